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
    __device__ __forceinline__ static bool get(const RowKPM::Cols& c, size_t g) { return c.m[g] != 0; }
};
template <int W, int KW>
struct MarkAt<RowRec<W, KW>> {
    __device__ __forceinline__ static bool get(const typename RowRec<W, KW>::Cols& c, size_t g)
    {
        return (((c.w[0][g] >> c.mark_bit) & 1ull) != 0) != (c.mark_inv != 0);
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

// calls f(std::integral_constant<int, v>) for a runtime v in [0, N)
template <int I, int N, class F>
__device__ __forceinline__ void static_switch(int v, F& f)
{
    if constexpr (I < N) {
        if (v == I)
            f(std::integral_constant<int, I> {});
        else
            static_switch<I + 1, N>(v, f);
    }
}

// exchange decision for the pair (a at the lower index, b): ascending swaps
// iff a > b, descending iff a < b (strict, as include/cuda/sort.cuh:31-40)
template <class R>
__device__ __forceinline__ bool need_swap(const R& a, const R& b, bool desc, const typename R::Cols& c)
{
    if constexpr (R::FULL_KEY) {
        // every field is compared, so equal rows are identical and swapping
        // them is a no-op: one comparison decides both directions
        return R::gt(a, b, c) != desc;
    } else {
        return desc ? R::gt(b, a, c) : R::gt(a, b, c);
    }
}

template <class R, int LOG_NT, int LOG_E>
struct Net {
    using TL = Tile<LOG_NT, LOG_E>;
    using Cols = typename R::Cols;
    static constexpr int E = TL::E;
    static constexpr int LT = TL::LOG_T;
    static constexpr int T = TL::T;
    static constexpr int S0 = LT - LOG_E; // load/store layout (lanes <-> rows 0..31)
    static constexpr int NS = S0 + 1;     // layouts 0..S0

    static constexpr size_t smem_rows() { return ((size_t)T * R::SMEM_BYTES + 15) & ~(size_t)15; }
    static constexpr size_t smem_bytes_sort() { return smem_rows(); }
    static constexpr size_t smem_bytes_compact() { return smem_rows() + (size_t)T * 4 + 33 * 4; }

    // thread part of the local row index in layout S
    template <int S>
    __device__ __forceinline__ static int tidpart()
    {
        const int tid = threadIdx.x;
        return (tid & ((1 << S) - 1)) | ((tid >> S) << (S + LOG_E));
    }

    template <int S>
    __device__ __forceinline__ static void sstore_all(const R (&v)[E], char* sm)
    {
        const int tp = tidpart<S>();
#pragma unroll
        for (int e = 0; e < E; e++)
            R::sstore(sm, T, TL::swz(tp | (e << S)), v[e]);
    }
    template <int S>
    __device__ __forceinline__ static void sload_all(R (&v)[E], const char* sm)
    {
        const int tp = tidpart<S>();
#pragma unroll
        for (int e = 0; e < E; e++)
            v[e] = R::sload(sm, T, TL::swz(tp | (e << S)));
    }

    // re-layout the tile from layout `from` to layout `to` through smem
    __device__ __forceinline__ static void transpose(R (&v)[E], int from, int to, char* sm)
    {
        __syncthreads();
        auto st = [&](auto sc) { sstore_all<decltype(sc)::value>(v, sm); };
        static_switch<0, NS>(from, st);
        __syncthreads();
        auto ld = [&](auto sc) { sload_all<decltype(sc)::value>(v, sm); };
        static_switch<0, NS>(to, ld);
    }

    // ---- bitonic compare-exchange on register bit Q in layout S -----------
    template <int S, int Q>
    __device__ __forceinline__ static void bitonic_level(R (&v)[E], const Cols& c, int K, bool dconst, bool asc_c)
    {
        const int tp = tidpart<S>();
        const bool tdesc = ((tp >> K) & 1) != 0; // thread part of the direction bit
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (e & (1 << Q))
                continue;
            const int e2 = e | (1 << Q);
            const bool desc = dconst ? !asc_c : (tdesc | ((((e << S) >> K) & 1) != 0));
            const bool sw = need_swap(v[e], v[e2], desc, c);
            const R a = R::select(sw, v[e2], v[e]);
            const R b = R::select(sw, v[e], v[e2]);
            v[e] = a;
            v[e2] = b;
        }
    }

    __device__ __forceinline__ static void bitonic(int s, int q, R (&v)[E], const Cols& c, int K, bool dconst,
                                                   bool asc_c)
    {
        auto fs = [&](auto sc) {
            constexpr int S = decltype(sc)::value;
            auto fq = [&](auto qc) { bitonic_level<S, decltype(qc)::value>(v, c, K, dconst, asc_c); };
            static_switch<0, LOG_E>(q, fq);
        };
        static_switch<0, NS>(s, fs);
    }

    // ---- ORCompact exchange (tile-local level, block size 2^(b+1)) --------
    // Pair (l, l + 2^b) inside block S; the block's offset is P[S] mod 2^(b+1)
    // and its left-half mark count is P[S + 2^b] - P[S] (P = exclusive prefix
    // of the original marks; block counts are invariant under the
    // permutations of lower levels).
    template <int S, int Q>
    __device__ __forceinline__ static void compact_level_tile(R (&v)[E], const Cols& c, int b, uint32_t p_tile,
                                                              const uint32_t* pre)
    {
        const int tp = tidpart<S>();
        const uint32_t half = 1u << b;
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (e & (1 << Q))
                continue;
            const int e2 = e | (1 << Q);
            const int l = tp | (e << S);
            const int blk = l & ~(int)(2 * half - 1);
            const uint32_t ps = p_tile + pre[blk];
            bool sw;
            if (b == 0) {
                // compact_offset, n == 2 (algorithms.c:123-128)
                const bool ml = MarkOf<R>::get(v[e], c), mr = MarkOf<R>::get(v[e2], c);
                sw = ((!ml) & mr) != ((ps & 1u) == 1u);
            } else {
                // compact_offset, n > 2 (algorithms.c:130-152)
                const uint32_t left = pre[blk + half] - pre[blk];
                const uint32_t off = ps & (2 * half - 1);
                const uint32_t i = (uint32_t)(l - blk);
                const bool sb = (((off & (half - 1)) + left) >= half) != (off >= half);
                sw = sb != (i >= ((off + left) & (half - 1)));
            }
            const R a = R::select(sw, v[e2], v[e]);
            const R bb = R::select(sw, v[e], v[e2]);
            v[e] = a;
            v[e2] = bb;
        }
    }

    template <int S, int Q>
    __device__ __forceinline__ static void compact_level_global(R (&v)[E], const Cols& c, int b,
                                                                const uint32_t* tile_prefix, int C, int b_lo,
                                                                size_t cta_bits)
    {
        const int tp = tidpart<S>();
        const uint64_t half = 1ull << b;
#pragma unroll
        for (int e = 0; e < E; e++) {
            if (e & (1 << Q))
                continue;
            const int e2 = e | (1 << Q);
            const int l = tp | (e << S);
            const uint64_t g = (uint64_t)(l & ((1 << C) - 1)) | ((uint64_t)(l >> C) << b_lo) | cta_bits;
            const uint64_t blk = g & ~(2 * half - 1);
            const uint32_t ps = tile_prefix[blk >> LT];
            const uint32_t pm = tile_prefix[(blk + half) >> LT];
            const uint64_t left = pm - ps;
            const uint64_t off = ps & (2 * half - 1);
            const uint64_t i = g - blk;
            const bool sb = (((off & (half - 1)) + left) >= half) != (off >= half);
            const bool sw = sb != (i >= ((off + left) & (half - 1)));
            const R a = R::select(sw, v[e2], v[e]);
            const R bb = R::select(sw, v[e], v[e2]);
            v[e] = a;
            v[e2] = bb;
        }
    }

    // ---- one pass over one tile (CTA `cta`) --------------------------------
    // SORT = true compiles only the bitonic pass kinds, false only ORCompact.
    template <bool SORT>
    __device__ static void run(const Cols& c, const NetGeom& g, const NetPass& p, const uint32_t* tile_prefix,
                               int cta, char* sm)
    {
        const int tid = threadIdx.x;
        const size_t Np = (size_t)1 << g.logN;
        const bool is_global = (p.kind == P_SORT_GLOBAL) || (p.kind == P_COMPACT_GLOBAL);
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
        {
            auto ld = [&](auto sc) {
                constexpr int S = decltype(sc)::value;
                const int tp = tidpart<S>();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const size_t gi = gidx(tp | (e << S));
                    if (first)
                        v[e] = (gi < g.n) ? R::load(c, gi) : R::pad(c);
                    else
                        v[e] = R::load(c, gi);
                }
            };
            static_switch<0, NS>(s, ld);
        }

        if constexpr (SORT) {
        if (p.kind == P_SORT_TILE) {
            for (int K = 1; K <= p.K; K++) {
                const bool dconst = K >= LT;
                const bool asc_c = ((cta_bits >> K) & 1) == 0;
                for (int b = K - 1; b >= 0; b--) {
                    if (b < s || b >= s + LOG_E) {
                        const int ns = window_down(b, LOG_E, LT);
                        transpose(v, s, ns, sm);
                        s = ns;
                    }
                    bitonic(s, b - s, v, c, K, dconst, asc_c);
                }
            }
        } else if (p.kind == P_SORT_MERGE) {
            const bool asc_c = ((cta_bits >> p.K) & 1) == 0;
            for (int b = LT - 1; b >= 0; b--) {
                if (b < s || b >= s + LOG_E) {
                    const int ns = window_down(b, LOG_E, LT);
                    transpose(v, s, ns, sm);
                    s = ns;
                }
                bitonic(s, b - s, v, c, p.K, true, asc_c);
            }
        } else if (p.kind == P_SORT_GLOBAL) {
            const bool asc_c = ((gidx(0) >> p.K) & 1) == 0;
            for (int b = p.b_hi; b >= b_lo; b--) {
                const int lp = C + (b - b_lo);
                if (lp < s || lp >= s + LOG_E) {
                    int ns = window_down(lp, LOG_E, LT);
                    ns = ns < smin ? smin : ns;
                    transpose(v, s, ns, sm);
                    s = ns;
                }
                bitonic(s, lp - s, v, c, p.K, true, asc_c);
            }
        }
        } else {
        if (p.kind == P_COMPACT_TILE) {
            // prefix of the original marks over the tile, in local-index order
            uint32_t* pre = reinterpret_cast<uint32_t*>(sm + smem_rows());
            uint32_t* tmp = pre + T;
            transpose(v, s, 0, sm);
            s = 0;
            uint32_t cnt = 0, m[E];
#pragma unroll
            for (int e = 0; e < E; e++) {
                m[e] = cnt;
                cnt += MarkOf<R>::get(v[e], c) ? 1u : 0u;
            }
            uint32_t total;
            const uint32_t base = block_exclusive_scan(cnt, tmp, &total);
            const int tp0 = tidpart<0>();
#pragma unroll
            for (int e = 0; e < E; e++)
                pre[tp0 | e] = base + m[e];
            __syncthreads();
            const uint32_t p_tile = tile_prefix[cta];
            for (int b = 0; b < p.K; b++) {
                if (b < s || b >= s + LOG_E) {
                    const int ns = window_up(b, LOG_E, LT);
                    transpose(v, s, ns, sm);
                    s = ns;
                }
                auto fs = [&](auto sc) {
                    constexpr int S = decltype(sc)::value;
                    auto fq = [&](auto qc) { compact_level_tile<S, decltype(qc)::value>(v, c, b, p_tile, pre); };
                    static_switch<0, LOG_E>(b - S, fq);
                };
                static_switch<0, NS>(s, fs);
            }
        } else { // P_COMPACT_GLOBAL
            for (int b = b_lo; b <= p.b_hi; b++) {
                const int lp = C + (b - b_lo);
                if (lp < s || lp >= s + LOG_E) {
                    int ns = window_up(lp, LOG_E, LT);
                    ns = ns < smin ? smin : ns;
                    transpose(v, s, ns, sm);
                    s = ns;
                }
                auto fs = [&](auto sc) {
                    constexpr int S = decltype(sc)::value;
                    auto fq = [&](auto qc) {
                        compact_level_global<S, decltype(qc)::value>(v, c, b, tile_prefix, C, b_lo, cta_bits);
                    };
                    static_switch<0, LOG_E>(lp - S, fq);
                };
                static_switch<0, NS>(s, fs);
            }
        }
        }

        if (s < 5) {
            transpose(v, s, S0, sm);
            s = S0;
        }
        {
            auto stf = [&](auto sc) {
                constexpr int S = decltype(sc)::value;
                const int tp = tidpart<S>();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const size_t gi = gidx(tp | (e << S));
                    if (gi < Np)
                        R::store(c, gi, v[e]);
                }
            };
            static_switch<0, NS>(s, stf);
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
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
        const size_t gi = base + i;
        const bool in = gi < n;
        const size_t gs = in ? gi : 0; // every row index is public: read row 0 for pads
        cnt += (in & MarkAt<R>::get(c, gs)) ? 1u : 0u;
    }
    uint32_t total;
    block_exclusive_scan(cnt, tmp, &total);
    if (threadIdx.x == 0)
        counts[cta] = total;
}

// exclusive scan of the tile counts into prefix[0..ntiles]; one CTA
__device__ __forceinline__ void scan_tiles(const uint32_t* counts, int ntiles, uint32_t* prefix, uint64_t* d_count,
                                           uint32_t* tmp)
{
    uint32_t carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const uint32_t x = i < ntiles ? counts[i] : 0u;
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
