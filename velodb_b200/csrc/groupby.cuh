// Filter + group-by over a lineitem-shaped fact table: record layouts, the
// aggregate definition, the predicate/pack step and the scratch layout, shared
// by the plain pipeline (groupby.cu) and the persistent command queue
// (dq_kernel.cu).  The pipeline itself is described in groupby.cu.
#pragma once

#include "common.hpp"
#include "network.cuh"
#include "segagg.cuh"

namespace velo {

constexpr uint64_t LI_KEYMASK = 0xFFFF800000000000ull;
constexpr int LI_LT = 12; // 4096-row tiles for sort and compaction (CTA shape: Tile12)
constexpr int LI_FIELD_BITS = 15;
// global passes fuse up to 8 levels: 16 contiguous rows of 8-byte words are a
// whole 128-byte line, so 2^4-row segments keep the loads coalesced
constexpr int LI_LMAX = LI_LT - 4 < 8 ? LI_LT - 4 : 8;

// decoding parameters of the two-word layout (public: from the predicate)
struct LiParams {
    int32_t qty_lo;
    int32_t disc_lo;
    uint32_t qbits;
    uint32_t pad_;
};

template <int NW>
struct LineitemAgg {
    static constexpr int W = NW;
    static constexpr int V = 5; // count, sum qty, sum price, sum price*(100-disc), sum price*(100-disc)*(100+tax)
    using Params = LiParams;
    __device__ __forceinline__ static uint64_t key(const uint64_t* w) { return w[0] & LI_KEYMASK; }
    __device__ __forceinline__ static bool valid(const uint64_t* w) { return (w[0] >> 63) == 0; }
    __device__ __forceinline__ static void values(const uint64_t* w, int64_t (&v)[V], const Params& prm)
    {
        const bool ok = valid(w);
        int64_t qty, disc, tax;
        if constexpr (W == 3) {
            qty = (int64_t)(int32_t)(uint32_t)w[0];
            disc = (int64_t)(int32_t)(uint32_t)(w[2] >> 32);
            tax = (int64_t)(int32_t)(uint32_t)w[2];
        } else {
            const uint32_t f = (uint32_t)(w[0] >> 32) & ((1u << LI_FIELD_BITS) - 1u);
            qty = (int64_t)prm.qty_lo + (int64_t)(f & ((1u << prm.qbits) - 1u));
            disc = (int64_t)prm.disc_lo + (int64_t)(f >> prm.qbits);
            tax = (int64_t)(int32_t)(uint32_t)w[0];
        }
        const int64_t price = (int64_t)w[1];
        const int64_t dp = price * (100 - disc);
        v[0] = ok ? 1 : 0;
        v[1] = ok ? qty : 0;
        v[2] = ok ? price : 0;
        v[3] = ok ? dp : 0;
        v[4] = ok ? dp * (100 + tax) : 0;
    }
    __device__ __forceinline__ static int64_t out_key_from(uint64_t key) { return (int64_t)((key >> 47) & 0xFFFF); }
};

template <int W>
struct LiTypes {
    static constexpr int W_ = W;
    // ordered on the high half of word 0: the group key (bits 63:47) then
    // payload bits, a refinement of key order; the group-by sums over ties, so
    // the order inside a group is irrelevant
    using Rec = RowRec<W, 1, false, KEY_HI32>;
    using Agg = LineitemAgg<W>;
    using Seg = SegAgg<Agg>;
};
constexpr int LI_V = 5;

struct LiCols {
    const int32_t* qty;
    const int64_t* price;
    const int32_t* disc;
    const int32_t* tax;
    const int32_t* ship;
    const uint8_t* f1;
    const uint8_t* f2;
};

// predicate + pack of tile `blk` (2^lt rows) and the tile's pass count;
// tmp: 33 words of shared memory
template <int W>
__device__ __forceinline__ void li_pack_tile(const LiCols& c, const velo_lineitem_pred& p, const LiParams& prm,
                                             size_t n, size_t n_rec, int lt, uint64_t* w0, uint64_t* w1, uint64_t* w2,
                                             uint32_t* counts, size_t blk, uint32_t* tmp)
{
    const size_t base = blk << lt;
    const int T = 1 << lt;
    uint32_t cnt = 0;
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
        const size_t g = base + i;
        if (g >= n_rec)
            break;
        VELO_TRACE_AT(TS_LI_OUT, w0 + g);
        uint64_t r0 = ~0ull, r1 = ~0ull, r2 = ~0ull;
        if (g < n) {
            VELO_TRACE_AT(TS_LI_IN, c.qty + g);
            const int32_t q = c.qty[g], d = c.disc[g], t = c.tax[g], s = c.ship[g];
            const int64_t pr = c.price[g];
            const uint8_t a = c.f1[g], b = c.f2[g];
            const bool ok = (s >= p.ship_lo) & (s <= p.ship_hi) & (d >= p.disc_lo) & (d <= p.disc_hi) & (q >= p.qty_lo)
                & (q <= p.qty_hi);
            const uint64_t key = ((uint64_t)(!ok) << 63) | ((uint64_t)a << 55) | ((uint64_t)b << 47);
            if constexpr (W == 3) {
                r0 = key | (uint64_t)(uint32_t)q;
                r2 = ((uint64_t)(uint32_t)d << 32) | (uint64_t)(uint32_t)t;
            } else {
                const uint32_t f = ((uint32_t)(q - prm.qty_lo) | ((uint32_t)(d - prm.disc_lo) << prm.qbits))
                    & ((1u << LI_FIELD_BITS) - 1u);
                r0 = key | ((uint64_t)f << 32) | (uint64_t)(uint32_t)t;
            }
            r1 = (uint64_t)pr;
            cnt += ok ? 1u : 0u;
        }
        w0[g] = r0;
        w1[g] = r1;
        if constexpr (W == 3)
            w2[g] = r2;
    }
    uint32_t total;
    block_exclusive_scan(cnt, tmp, &total);
    if (threadIdx.x == 0)
        counts[blk] = total;
}

struct LiScratch {
    uint64_t* w[3];
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* d_rows;
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    int64_t* tile_out;
    uint64_t* n_groups;
    size_t bytes;
    size_t n_rec;
    int ntiles_c;
    int ntiles_s;
};

// Partition of the scratch buffer (offsets 256-byte aligned).
inline LiScratch li_layout(char* base, size_t n, uint32_t G)
{
    LiScratch s {};
    const size_t np = next_pow2(n);
    size_t n_rec = np;
    if (n_rec < (size_t)SEG_TS)
        n_rec = SEG_TS;
    if (n_rec < ((size_t)1 << LI_LT))
        n_rec = (size_t)1 << LI_LT;
    s.n_rec = n_rec;
    s.ntiles_c = (int)(n_rec >> LI_LT);
    s.ntiles_s = (int)(n_rec / SEG_TS);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes, 256);
        return p;
    };
    for (int i = 0; i < 3; i++)
        s.w[i] = reinterpret_cast<uint64_t*>(take(n_rec * 8));
    // room for the tile counts of 2^(LI_LT-1)-row tiles: the persistent
    // command queue compacts three-word records in 2048-row tiles
    const size_t cnt_tiles = n_rec >> (LI_LT - 1);
    s.counts = reinterpret_cast<uint32_t*>(take(cnt_tiles * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take((cnt_tiles + 1) * 4));
    s.d_rows = reinterpret_cast<uint64_t*>(take(8));
    s.aggs = reinterpret_cast<SegTileAgg*>(take((size_t)s.ntiles_s * sizeof(SegTileAgg)));
    s.runs = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * LI_V * 8));
    s.carry = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * LI_V * 8));
    s.tail_prefix = reinterpret_cast<uint32_t*>(take((size_t)s.ntiles_s * 4));
    s.tile_out = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * G * (1 + LI_V) * 8));
    s.n_groups = reinterpret_cast<uint64_t*>(take(8));
    s.bytes = off;
    return s;
}

// bits needed for the offsets 0..hi-lo of a band (0 for an empty or one-value band)
inline uint32_t band_bits(int32_t lo, int32_t hi)
{
    const int64_t w = (int64_t)hi - (int64_t)lo;
    uint32_t b = 0;
    while (w > 0 && b < 33 && ((int64_t)1 << b) <= w)
        b++;
    return b;
}

} // namespace velo
