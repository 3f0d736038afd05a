// Oblivious filter + group-by over a lineitem-shaped fact table.
//
// Pipeline (all on the device, one stream, no host round trip unless the
// caller asks to reveal the filtered count as the reference does):
//   1. pack     predicate (conjunctive ranges, the pushed-down WHERE of
//               src/operator/seq_scan_operator.cpp:38-45 evaluated on the GPU)
//               and packing of each row into a 3-word record; per-tile counts
//               of the rows that pass
//   2. compact  ORCompact of the records (passing rows first, in input order)
//               -- replaces FilterCompactionOperator's scatter/gather
//               (src/operator/filter_compaction_operator.cpp:65-184)
//   3. sort     bitonic network on the group key (flag1, flag2)
//   4. segagg   segmented sums per group with a public output bound
//               (obliviator/operator_2/enclave/scalable_oblivious_join.c:221-262)
// Record layouts (u64 words).  Three words in general:
//   w0 = [63] row fails the filter | [62:55] flag1 | [54:47] flag2 | [31:0] quantity
//   w1 = extended price (int64, cents)
//   w2 = discount (int32) << 32 | tax (int32)
// Two words when the predicate's quantity and discount bands are narrow: a
// passing row's quantity and discount lie inside those public bands, so each
// is stored as its offset from the band's lower bound in the 15 bits between
// the key and the tax (qbits + dbits <= 15, both from the public predicate):
//   w0 = [63] fails | [62:55] flag1 | [54:47] flag2
//        | [46:32] (disc - disc_lo) << qbits | (qty - qty_lo) | [31:0] tax
//   w1 = extended price
// The layout is chosen from the predicate alone, never from the data.  The
// group key is w0[63:47]; the sort orders on w0[63:32], which refines the key
// order; failing rows sort after every passing row.
#include "net_impl.cuh"
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

template <int W>
__global__ void __launch_bounds__(256) k_li_pack(LiCols c, velo_lineitem_pred p, LiParams prm, size_t n,
                                                 size_t n_rec, int lt, uint64_t* w0, uint64_t* w1, uint64_t* w2,
                                                 uint32_t* counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_li_pack"));
    __shared__ uint32_t tmp[33];
    const size_t base = (size_t)blockIdx.x << lt;
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
        counts[blockIdx.x] = total;
}

template <int W>
__global__ void __launch_bounds__(SEG_THREADS) k_seg_summary(typename LiTypes<W>::Rec::Cols c, SegTileAgg* aggs,
                                                             int64_t* runs, LiParams prm)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_summary"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::tile_summary(c.w, blockIdx.x, aggs, runs, prm, sm);
}

template <int W>
__global__ void __launch_bounds__(1024) k_seg_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                      int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_carries"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

template <int W>
__global__ void __launch_bounds__(SEG_THREADS) k_seg_emit(typename LiTypes<W>::Rec::Cols c, int ntiles,
                                                          const SegTileAgg* aggs, const int64_t* carry_in,
                                                          const uint32_t* tail_prefix, int G, int64_t* tile_out,
                                                          LiParams prm)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_emit"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::emit(c.w, blockIdx.x, ntiles, aggs, carry_in, tail_prefix, G, tile_out, prm, sm);
}

// CTA q of G*(1+V): output word q; CTA 0 also writes the two counts
__global__ void __launch_bounds__(SEG_THREADS) k_seg_finish(const int64_t* tile_out, int ntiles, int G, int64_t* out,
                                                            const uint64_t* d_rows, const uint64_t* n_groups,
                                                            uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_finish"));
    LiTypes<3>::Seg::finish(tile_out, ntiles, G, out);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d_counts[0] = *d_rows;
        d_counts[1] = *n_groups;
    }
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
static LiScratch li_layout(char* base, size_t n, uint32_t G)
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
    s.counts = reinterpret_cast<uint32_t*>(take((size_t)s.ntiles_c * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take(((size_t)s.ntiles_c + 1) * 4));
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

template <int W>
static velo_status seg_smem_attrs()
{
    using Seg = typename LiTypes<W>::Seg;
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev])
        return VELO_OK;
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_summary<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Seg::SMEM_IN),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_emit<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Seg::SMEM_IN),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_carries<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(LI_V * 1024 * 8 + 2 * 1024 * 4)),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
    return VELO_OK;
}

// bits needed for the offsets 0..hi-lo of a band (0 for an empty or one-value band)
static uint32_t band_bits(int32_t lo, int32_t hi)
{
    const int64_t w = (int64_t)hi - (int64_t)lo;
    uint32_t b = 0;
    while (w > 0 && b < 33 && ((int64_t)1 << b) <= w)
        b++;
    return b;
}

template <int W>
static velo_status run_groupby(const LiScratch& s, const LiCols& c, size_t n, const velo_lineitem_pred& pred,
                               const LiParams& prm, uint32_t group_bound, uint32_t flags, int64_t* d_out,
                               uint64_t* d_counts, cudaStream_t st)
{
    using Rec = typename LiTypes<W>::Rec;
    using Seg = typename LiTypes<W>::Seg;
    velo_status rc = seg_smem_attrs<W>();
    if (rc != VELO_OK)
        return rc;
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    StageTimer tm(st);

    // 1. predicate + pack (+ per-tile pass counts)
    k_li_pack<W><<<s.ntiles_c, 256, 0, st>>>(c, pred, prm, n, s.n_rec, LI_LT, s.w[0], s.w[1], s.w[2], s.counts);
    const int ntiles_np = logN > LI_LT ? 1 << (logN - LI_LT) : 1;
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntiles_np, s.prefix, s.d_rows);
    VELO_CUDA_TRY(cudaGetLastError(), "pack launch");
    tm.mark();

    typename Rec::Cols rc3;
    for (int i = 0; i < W; i++) {
        rc3.w[i] = s.w[i];
        rc3.pad[i] = ~0ull;
    }
    rc3.mask[0] = LI_KEYMASK;
    rc3.mark_bit = 63;
    rc3.mark_inv = 1;
    rc3.mark_word = 0;

    // 2. ORCompact over the next_pow2(n) records
    {
        std::vector<NetPass> passes;
        plan_compact(logN, LI_LT, LI_LMAX, passes);
        NetGeom g { np, logN, 0 };
        rc = launch_net12<Rec>(rc3, g, passes, s.prefix, st);
        if (rc != VELO_OK)
            return rc;
    }
    tm.mark();
    // 3. sort by group key: all next_pow2(n) rows, or -- when the caller
    // reveals the filtered count like the reference operator -- only
    // next_pow2(count) rows
    int logS = logN;
    if (flags & VELO_REVEAL_COUNT) {
        uint64_t cnt = 0;
        VELO_CUDA_TRY(cudaMemcpyAsync(&cnt, s.d_rows, 8, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        VELO_CUDA_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        logS = ilog2_floor(next_pow2(cnt ? cnt : 1));
    }
    rc = launch_sort_records<Rec>(rc3, logS, st);
    if (rc != VELO_OK)
        return rc;
    tm.mark();
    // 4. segmented sums with public output bound
    size_t nseg = (size_t)1 << logS;
    if (nseg < (size_t)SEG_TS)
        nseg = SEG_TS;
    const int ntiles_s = (int)(nseg / SEG_TS);
    k_seg_summary<W><<<ntiles_s, SEG_THREADS, Seg::SMEM_IN, st>>>(rc3, s.aggs, s.runs, prm);
    k_seg_carries<W><<<1, 1024, LI_V * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, ntiles_s, s.carry,
                                                                      s.tail_prefix, s.n_groups);
    k_seg_emit<W><<<ntiles_s, SEG_THREADS, Seg::SMEM_IN, st>>>(rc3, ntiles_s, s.aggs, s.carry, s.tail_prefix,
                                                              (int)group_bound, s.tile_out, prm);
    k_seg_finish<<<group_bound * (1 + LI_V), SEG_THREADS, 0, st>>>(s.tile_out, ntiles_s, (int)group_bound, d_out,
                                                                   s.d_rows, s.n_groups, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by launch");
    tm.mark();
    tm.finish();
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_filter_groupby_scratch_bytes(size_t n, uint32_t group_bound)
{
    if (group_bound == 0 || group_bound > SEG_MAX_G)
        return 0;
    return li_layout(nullptr, n, group_bound).bytes;
}

extern "C" velo_status velo_filter_groupby(const velo_lineitem* cols, size_t n, const velo_lineitem_pred* pred,
                                           uint32_t group_bound, uint32_t flags, int64_t* d_out, uint64_t* d_counts,
                                           void* d_scratch, size_t scratch_bytes, void* stream)
{
    if (!cols || !pred || !d_out || !d_counts)
        return einval("velo_filter_groupby: null argument");
    if (group_bound == 0 || group_bound > SEG_MAX_G)
        return einval("velo_filter_groupby: group_bound must be 1..16");
    if (n == 0 || next_pow2(n) > ((size_t)1 << MAX_LOGN))
        return einval("velo_filter_groupby: n must be 1..2^31");
    if (!cols->qty || !cols->price || !cols->disc || !cols->tax || !cols->shipdate || !cols->flag1 || !cols->flag2)
        return einval("velo_filter_groupby: null column");
    LiScratch s = li_layout(static_cast<char*>(d_scratch), n, group_bound);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_filter_groupby: scratch must hold velo_filter_groupby_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    LiCols c { cols->qty, cols->price, cols->disc, cols->tax, cols->shipdate, cols->flag1, cols->flag2 };
    LiParams prm { pred->qty_lo, pred->disc_lo, band_bits(pred->qty_lo, pred->qty_hi), 0 };
    const uint32_t dbits = band_bits(pred->disc_lo, pred->disc_hi);
    if (prm.qbits + dbits <= (uint32_t)LI_FIELD_BITS)
        return run_groupby<2>(s, c, n, *pred, prm, group_bound, flags, d_out, d_counts, st);
    return run_groupby<3>(s, c, n, *pred, prm, group_bound, flags, d_out, d_counts, st);
}
