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
// Record layout (u64 words):
//   w0 = [63] row fails the filter | [62:55] flag1 | [54:47] flag2 | [31:0] quantity
//   w1 = extended price (int64, cents)
//   w2 = discount (int32) << 32 | tax (int32)
// The sort key is w0[63:47]; failing rows sort after every passing row.
#include "net_impl.cuh"
#include "segagg.cuh"

namespace velo {

// the group-by consumer sums over ties, so their arrangement is irrelevant
using LiRec = RowRec<3, 1, false>;
constexpr uint64_t LI_KEYMASK = 0xFFFF800000000000ull;
constexpr int LI_LOG_NT = 8, LI_LOG_E = 4; // 4096-row tiles for sort and compaction
constexpr int LI_LT = LI_LOG_NT + LI_LOG_E;

struct LineitemAgg {
    static constexpr int W = 3;
    static constexpr int V = 5; // count, sum qty, sum price, sum price*(100-disc), sum price*(100-disc)*(100+tax)
    __device__ __forceinline__ static uint64_t key(const uint64_t* w) { return w[0] & LI_KEYMASK; }
    __device__ __forceinline__ static bool valid(const uint64_t* w) { return (w[0] >> 63) == 0; }
    __device__ __forceinline__ static void values(const uint64_t* w, int64_t (&v)[V])
    {
        const bool ok = valid(w);
        const int64_t qty = (int64_t)(int32_t)(uint32_t)w[0];
        const int64_t price = (int64_t)w[1];
        const int64_t disc = (int64_t)(int32_t)(uint32_t)(w[2] >> 32);
        const int64_t tax = (int64_t)(int32_t)(uint32_t)w[2];
        const int64_t dp = price * (100 - disc);
        v[0] = ok ? 1 : 0;
        v[1] = ok ? qty : 0;
        v[2] = ok ? price : 0;
        v[3] = ok ? dp : 0;
        v[4] = ok ? dp * (100 + tax) : 0;
    }
    __device__ __forceinline__ static int64_t out_key_from(uint64_t key) { return (int64_t)((key >> 47) & 0xFFFF); }
};

using LiSeg = SegAgg<LineitemAgg>;

struct LiCols {
    const int32_t* qty;
    const int64_t* price;
    const int32_t* disc;
    const int32_t* tax;
    const int32_t* ship;
    const uint8_t* f1;
    const uint8_t* f2;
};

__global__ void __launch_bounds__(256) k_li_pack(LiCols c, velo_lineitem_pred p, size_t n, size_t n_rows, int lt,
                                                 uint64_t* w0, uint64_t* w1, uint64_t* w2, uint32_t* counts)
{
    __shared__ uint32_t tmp[33];
    const size_t base = (size_t)blockIdx.x << lt;
    const int T = 1 << lt;
    uint32_t cnt = 0;
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
        const size_t g = base + i;
        if (g >= n_rows)
            break;
        uint64_t r0 = ~0ull, r1 = ~0ull, r2 = ~0ull;
        if (g < n) {
            const int32_t q = c.qty[g], d = c.disc[g], t = c.tax[g], s = c.ship[g];
            const int64_t pr = c.price[g];
            const uint8_t a = c.f1[g], b = c.f2[g];
            const bool ok = (s >= p.ship_lo) & (s <= p.ship_hi) & (d >= p.disc_lo) & (d <= p.disc_hi) & (q >= p.qty_lo)
                & (q <= p.qty_hi);
            r0 = ((uint64_t)(!ok) << 63) | ((uint64_t)a << 55) | ((uint64_t)b << 47) | (uint64_t)(uint32_t)q;
            r1 = (uint64_t)pr;
            r2 = ((uint64_t)(uint32_t)d << 32) | (uint64_t)(uint32_t)t;
            cnt += ok ? 1u : 0u;
        }
        w0[g] = r0;
        w1[g] = r1;
        w2[g] = r2;
    }
    uint32_t total;
    block_exclusive_scan(cnt, tmp, &total);
    if (threadIdx.x == 0)
        counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SEG_THREADS) k_seg_summary(LiRec::Cols c, SegTileAgg* aggs, int64_t* runs)
{
    extern __shared__ __align__(16) char sm[];
    LiSeg::tile_summary(c.w, blockIdx.x, aggs, runs, sm);
}

__global__ void __launch_bounds__(1024) k_seg_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                      int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    extern __shared__ __align__(16) char sm[];
    LiSeg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

__global__ void __launch_bounds__(SEG_THREADS) k_seg_emit(LiRec::Cols c, int ntiles, const SegTileAgg* aggs,
                                                          const int64_t* carry_in, const uint32_t* tail_prefix,
                                                          int G, int64_t* tile_out)
{
    extern __shared__ __align__(16) char sm[];
    LiSeg::emit(c.w, blockIdx.x, ntiles, aggs, carry_in, tail_prefix, G, tile_out, sm);
}

__global__ void k_seg_finish(const int64_t* tile_out, int ntiles, int G, int64_t* out, const uint64_t* d_rows,
                             const uint64_t* n_groups, uint64_t* d_counts)
{
    LiSeg::finish(tile_out, ntiles, G, out);
    if (threadIdx.x == 0) {
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
    s.runs = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * LineitemAgg::V * 8));
    s.carry = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * LineitemAgg::V * 8));
    s.tail_prefix = reinterpret_cast<uint32_t*>(take((size_t)s.ntiles_s * 4));
    s.tile_out = reinterpret_cast<int64_t*>(take((size_t)s.ntiles_s * G * (1 + LineitemAgg::V) * 8));
    s.n_groups = reinterpret_cast<uint64_t*>(take(8));
    s.bytes = off;
    return s;
}

static velo_status seg_smem_attrs()
{
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev])
        return VELO_OK;
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_summary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LiSeg::SMEM),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_emit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LiSeg::SMEM),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_carries, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(LineitemAgg::V * 1024 * 8 + 2 * 1024 * 4)),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
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
    velo_status rc = seg_smem_attrs();
    if (rc != VELO_OK)
        return rc;
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);

    // 1. predicate + pack (+ per-tile pass counts)
    LiCols c { cols->qty, cols->price, cols->disc, cols->tax, cols->shipdate, cols->flag1, cols->flag2 };
    k_li_pack<<<s.ntiles_c, 256, 0, st>>>(c, *pred, n, s.n_rec, LI_LT, s.w[0], s.w[1], s.w[2], s.counts);
    const int ntiles_np = logN > LI_LT ? 1 << (logN - LI_LT) : 1;
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntiles_np, s.prefix, s.d_rows);
    VELO_CUDA_TRY(cudaGetLastError(), "pack launch");

    LiRec::Cols rc3;
    for (int i = 0; i < 3; i++) {
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
        plan_compact(logN, LI_LT, LI_LT - 5 < 8 ? LI_LT - 5 : 8, passes);
        NetGeom g { np, logN, 0 };
        rc = launch_net<LiRec, LI_LOG_NT, LI_LOG_E>(rc3, g, passes, s.prefix, st);
        if (rc != VELO_OK)
            return rc;
    }
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
    if (logS > 0) {
        std::vector<NetPass> passes;
        plan_sort(logS, LI_LT, LI_LT - 5 < 8 ? LI_LT - 5 : 8, passes);
        NetGeom g { (size_t)1 << logS, logS, 0 };
        rc = launch_net<LiRec, LI_LOG_NT, LI_LOG_E>(rc3, g, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
    }
    // 4. segmented sums with public output bound
    size_t nseg = (size_t)1 << logS;
    if (nseg < (size_t)SEG_TS)
        nseg = SEG_TS;
    const int ntiles_s = (int)(nseg / SEG_TS);
    k_seg_summary<<<ntiles_s, SEG_THREADS, LiSeg::SMEM, st>>>(rc3, s.aggs, s.runs);
    k_seg_carries<<<1, 1024, LineitemAgg::V * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, ntiles_s, s.carry,
                                                                                s.tail_prefix, s.n_groups);
    k_seg_emit<<<ntiles_s, SEG_THREADS, LiSeg::SMEM, st>>>(rc3, ntiles_s, s.aggs, s.carry, s.tail_prefix,
                                                           (int)group_bound, s.tile_out);
    k_seg_finish<<<1, 1024, 0, st>>>(s.tile_out, ntiles_s, (int)group_bound, d_out, s.d_rows, s.n_groups, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by launch");
    return VELO_OK;
}
