// Oblivious GROUP BY key with SUM / COUNT aggregates (velo_ogroupby).
//
// The reference engine has no aggregate operator (the plan node enum of
// include/planner/abstract_plan_node.hpp:31 names it, nothing implements it);
// the algorithm is the oblivious group-by of
// obliviator/operator_2/enclave/scalable_oblivious_join.c:105-262 (sort,
// forward segmented sum, group boundaries, compaction of one row per group),
// on the device:
//   1. pack     record = [63] row excluded (mask 0, or key out of range)
//               | order-preserving key in bits 62..0, then the sum columns
//   2. sort     bitonic network on the whole of word 0
//   3. segagg   segmented sums over the key runs (segagg.cuh); every row
//               writes a group record, valid on the last row of each run
//   4. compact  ORCompact of the group records: groups first, in key order
//   5. out      the first group_bound group records, decoded (zeros past the
//               number of groups)
// Every address depends only on n, group_bound and the key type.  INTEGER
// keys share word 0 with the exclusion bit.  BIGINT keys use all 64 bits of
// word 0 (key ^ 2^63), so their records carry the row's validity in a word of
// its own, sorted after the key: within a key the rows left out come first,
// so a key run ends on a valid row exactly when it holds one; their group
// records carry the group flag in a word of its own too (segagg FLAG_WORD).
#include "net_impl.cuh"
#include "segagg.cuh"

namespace velo {

constexpr int GB_LT = 12; // 4096-row tiles (CTA shape per record width: Tile12)
// up to 8 fused global levels: 16 contiguous rows of 8-byte words fill a line
constexpr int GB_LMAX = GB_LT - 4 < 8 ? GB_LT - 4 : 8;
constexpr uint64_t GB_EXCL = 1ull << 63;
constexpr int64_t GB_BIG = (int64_t)1 << 62;

// NS sum columns, CNT = 1 adds COUNT; V = NS + CNT aggregates
template <int NS, int CNT>
struct GbAgg {
    static constexpr int W = 1 + NS;
    static constexpr int V = NS + CNT;
    struct Params { };
    __device__ __forceinline__ static uint64_t key(const uint64_t* w) { return w[0]; }
    __device__ __forceinline__ static bool valid(const uint64_t* w) { return (w[0] & GB_EXCL) == 0; }
    __device__ __forceinline__ static void values(const uint64_t* w, int64_t (&v)[V], const Params&)
    {
        const bool ok = valid(w);
        int i = 0;
        if constexpr (CNT == 1)
            v[i++] = ok ? 1 : 0;
#pragma unroll
        for (int s = 0; s < NS; s++)
            v[i + s] = ok ? (int64_t)w[1 + s] : 0;
    }
    __device__ __forceinline__ static int64_t out_key_from(uint64_t key) { return (int64_t)(key & ~GB_EXCL); }
    __device__ __forceinline__ static uint64_t out_bits(uint64_t key) { return key & ~GB_EXCL; }
};

// BIGINT keys: records (key ^ 2^63, validity, sum 0, sum 1); aggregates
// (count, sum 0, sum 1) -- the ones not asked for are computed on zeros and
// dropped at the output
struct GbAggWide {
    static constexpr int W = 4;
    static constexpr int V = 3;
    static constexpr bool FLAG_WORD = true;
    struct Params { };
    __device__ __forceinline__ static uint64_t key(const uint64_t* w) { return w[0]; }
    __device__ __forceinline__ static bool valid(const uint64_t* w) { return (w[1] & 1ull) != 0; }
    __device__ __forceinline__ static void values(const uint64_t* w, int64_t (&v)[V], const Params&)
    {
        const bool ok = valid(w);
        v[0] = ok ? 1 : 0;
        v[1] = ok ? (int64_t)w[2] : 0;
        v[2] = ok ? (int64_t)w[3] : 0;
    }
    __device__ __forceinline__ static int64_t out_key_from(uint64_t key) { return (int64_t)(key ^ (1ull << 63)); }
    __device__ __forceinline__ static uint64_t out_bits(uint64_t key) { return key; }
};

// the per-tile run and carry arrays of the scratch hold 3 values a tile
static_assert(GbAggWide::V <= 3 && GbAgg<2, 0>::V <= 3 && GbAgg<1, 1>::V <= 3, "aggregates a tile in scratch");

struct GbTypesWide {
    using Agg = GbAggWide;
    using Seg = SegAgg<Agg>;
    using Rec = RowRec<4, 2, false, KEY_FULL>; // sorted on (key, validity)
    using Grp = RowRec<5, 1, false>;           // key, flag, count, sum 0, sum 1
};

template <int NS, int CNT>
struct GbTypes {
    using Agg = GbAgg<NS, CNT>;
    using Seg = SegAgg<Agg>;
    using Rec = RowRec<1 + NS, 1, false, KEY_FULL>;  // sorted on the whole of word 0
    using Grp = RowRec<1 + NS + CNT, 1, false>;      // group records, compaction only
};

struct GbIn {
    const void* keys;
    const int64_t* sums[2];
    const uint8_t* mask;
    uint32_t key_type;
};

__device__ __forceinline__ uint64_t gb_encode(const GbIn& in, size_t i, bool& ok)
{
    if (in.key_type == VELO_INTEGER) {
        const uint32_t k = static_cast<const uint32_t*>(in.keys)[i];
        return (uint64_t)(k ^ 0x80000000u) << 31;
    }
    const int64_t k = static_cast<const int64_t*>(in.keys)[i];
    ok = ok & (k >= -GB_BIG) & (k < GB_BIG);
    return (uint64_t)(k + GB_BIG) & ~GB_EXCL;
}

__device__ __forceinline__ int64_t gb_decode(uint32_t key_type, uint64_t bits)
{
    if (key_type == VELO_INTEGER)
        return (int64_t)(int32_t)((uint32_t)(bits >> 31) ^ 0x80000000u);
    return (int64_t)bits - GB_BIG;
}

template <int NS>
__global__ void __launch_bounds__(256) k_gb_pack(GbIn in, size_t n, size_t np, uint64_t* w0, uint64_t* w1,
                                                 uint64_t* w2, unsigned long long* d_rejected)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_pack"));
    __shared__ uint32_t tmp[33];
    uint32_t bad = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, np);
         i += (size_t)gridDim.x * blockDim.x) {
        uint64_t a = ~0ull, s0 = 0, s1 = 0;
        if (i < n) {
            bool in_range = true;
            const uint64_t enc = gb_encode(in, i, in_range);
            const bool take = in.mask ? in.mask[i] != 0 : true;
            bad += (take & !in_range) ? 1u : 0u;
            a = enc | ((take & in_range) ? 0ull : GB_EXCL);
            if constexpr (NS >= 1)
                s0 = (uint64_t)in.sums[0][i];
            if constexpr (NS >= 2)
                s1 = (uint64_t)in.sums[1][i];
        }
        w0[i] = a;
        if constexpr (NS >= 1)
            w1[i] = s0;
        if constexpr (NS >= 2)
            w2[i] = s1;
    }
    // one counter update per CTA at a fixed address
    uint32_t total;
    block_exclusive_scan(bad, tmp, &total);
    if (threadIdx.x == 0 && total)
        atomicAdd(d_rejected, (unsigned long long)total);
}

__global__ void __launch_bounds__(256) k_gb_pack_wide(GbIn in, int n_sums, size_t n, size_t np, uint64_t* w0,
                                                      uint64_t* w1, uint64_t* w2, uint64_t* w3)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_pack_wide"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, np);
         i += (size_t)gridDim.x * blockDim.x) {
        uint64_t k = ~0ull, f = 0, s0 = 0, s1 = 0;
        if (i < n) {
            k = (uint64_t) static_cast<const int64_t*>(in.keys)[i] ^ (1ull << 63);
            f = (in.mask ? in.mask[i] != 0 : true) ? 1ull : 0ull;
            s0 = n_sums >= 1 ? (uint64_t)in.sums[0][i] : 0ull;
            s1 = n_sums >= 2 ? (uint64_t)in.sums[1][i] : 0ull;
        }
        VELO_TRACE_AT(TS_ROW_STORE, w0 + i);
        w0[i] = k;
        w1[i] = f;
        w2[i] = s0;
        w3[i] = s1;
    }
}

__global__ void __launch_bounds__(SEG_THREADS) k_gbw_summary(GbTypesWide::Rec::Cols c, SegTileAgg* aggs, int64_t* runs)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gbw_summary"));
    extern __shared__ __align__(16) char sm[];
    GbTypesWide::Seg::tile_summary(c.w, blockIdx.x, aggs, runs, {}, sm);
}

__global__ void __launch_bounds__(1024) k_gbw_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                      int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gbw_carries"));
    extern __shared__ __align__(16) char sm[];
    GbTypesWide::Seg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

__global__ void __launch_bounds__(SEG_THREADS) k_gbw_emit_rows(GbTypesWide::Rec::Cols c, int ntiles,
                                                               const SegTileAgg* aggs, const int64_t* carry_in,
                                                               GbTypesWide::Grp::Cols g)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gbw_emit_rows"));
    extern __shared__ __align__(16) char sm[];
    GbTypesWide::Seg::emit_rows(c.w, blockIdx.x, ntiles, aggs, carry_in, g.w, {}, sm);
}

template <int NS, int CNT>
__global__ void __launch_bounds__(SEG_THREADS) k_gb_summary(typename GbTypes<NS, CNT>::Rec::Cols c, SegTileAgg* aggs,
                                                            int64_t* runs)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_summary"));
    extern __shared__ __align__(16) char sm[];
    GbTypes<NS, CNT>::Seg::tile_summary(c.w, blockIdx.x, aggs, runs, {}, sm);
}

template <int NS, int CNT>
__global__ void __launch_bounds__(1024) k_gb_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                     int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_carries"));
    extern __shared__ __align__(16) char sm[];
    GbTypes<NS, CNT>::Seg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

template <int NS, int CNT>
__global__ void __launch_bounds__(SEG_THREADS) k_gb_emit_rows(typename GbTypes<NS, CNT>::Rec::Cols c, int ntiles,
                                                              const SegTileAgg* aggs, const int64_t* carry_in,
                                                              typename GbTypes<NS, CNT>::Grp::Cols g)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_emit_rows"));
    extern __shared__ __align__(16) char sm[];
    GbTypes<NS, CNT>::Seg::emit_rows(c.w, blockIdx.x, ntiles, aggs, carry_in, g.w, {}, sm);
}

struct GbOut {
    int64_t* keys;
    int64_t* sums[2];
    int64_t* counts;
};

// group record words: g0 = [63] not a group | key bits, then the V aggregates
// in the Agg order (count first when present, then the sums)
template <int NS, int CNT>
__global__ void k_gb_out(const uint64_t* g0, const uint64_t* g1, const uint64_t* g2, size_t bound, uint32_t key_type,
                         GbOut out, const uint64_t* n_groups, const unsigned long long* rejected, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gb_out"));
    const uint64_t ng = *n_groups;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(j, bound);
         j += (size_t)gridDim.x * blockDim.x) {
        const bool ok = j < ng;
        const uint64_t a = g0[j];
        const uint64_t v[2] = { g1[j], NS + CNT > 1 ? g2[j] : 0ull };
        out.keys[j] = ok ? gb_decode(key_type, a & ~GB_EXCL) : 0;
        int i = 0;
        if constexpr (CNT == 1) {
            out.counts[j] = ok ? (int64_t)v[0] : 0;
            i = 1;
        }
#pragma unroll
        for (int s = 0; s < NS; s++)
            out.sums[s][j] = ok ? (int64_t)v[i + s] : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d_counts[0] = ng;
        d_counts[1] = *rejected;
    }
}

// wide group records: g[0] = key ^ 2^63, g[1] = flag, g[2] count, g[3..4] sums
struct GbwWords {
    const uint64_t* g[5];
};

__global__ void k_gbw_out(GbwWords g, size_t bound, int n_sums, int with_count, GbOut out,
                          const uint64_t* n_groups, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_gbw_out"));
    const uint64_t ng = *n_groups;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(j, bound);
         j += (size_t)gridDim.x * blockDim.x) {
        const bool ok = j < ng;
        VELO_TRACE_AT(TS_ROW_LOAD, g.g[0] + j);
        out.keys[j] = ok ? (int64_t)(g.g[0][j] ^ (1ull << 63)) : 0;
        if (with_count)
            out.counts[j] = ok ? (int64_t)g.g[2][j] : 0;
        for (int s = 0; s < n_sums; s++)
            out.sums[s][j] = ok ? (int64_t)g.g[3 + s][j] : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d_counts[0] = ng;
        d_counts[1] = 0;
    }
}

struct GbScratch {
    uint64_t* r[4];      // sort records
    uint64_t* g[5];      // group records
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* n_grp_rows;
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    uint64_t* n_groups;
    unsigned long long* rejected;
    size_t n_rec;
    size_t bytes;
};

static GbScratch gb_layout(char* base, size_t n)
{
    GbScratch s {};
    size_t np = next_pow2(n);
    if (np < ((size_t)1 << GB_LT))
        np = (size_t)1 << GB_LT;
    s.n_rec = np;
    const size_t ntc = np >> GB_LT, nts = np / SEG_TS;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes ? bytes : 1, 256);
        return p;
    };
    for (int i = 0; i < 4; i++)
        s.r[i] = reinterpret_cast<uint64_t*>(take(np * 8));
    for (int i = 0; i < 5; i++)
        s.g[i] = reinterpret_cast<uint64_t*>(take(np * 8));
    s.counts = reinterpret_cast<uint32_t*>(take(ntc * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take((ntc + 1) * 4));
    s.n_grp_rows = reinterpret_cast<uint64_t*>(take(8));
    s.aggs = reinterpret_cast<SegTileAgg*>(take(nts * sizeof(SegTileAgg)));
    // per tile: one value per aggregate (at most 3: the BIGINT path's
    // count and two sums)
    s.runs = reinterpret_cast<int64_t*>(take(nts * 3 * 8));
    s.carry = reinterpret_cast<int64_t*>(take(nts * 3 * 8));
    s.tail_prefix = reinterpret_cast<uint32_t*>(take(nts * 4));
    s.n_groups = reinterpret_cast<uint64_t*>(take(8));
    s.rejected = reinterpret_cast<unsigned long long*>(take(8));
    s.bytes = off;
    return s;
}

static unsigned gb_grid(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

template <int NS, int CNT>
static velo_status gb_run(const GbScratch& s, const GbIn& in, size_t n, size_t bound, GbOut out, uint64_t* d_counts,
                          cudaStream_t st)
{
    using T = GbTypes<NS, CNT>;
    using Seg = typename T::Seg;
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64 || !done[dev]) {
        VELO_CUDA_TRY(cudaFuncSetAttribute(k_gb_summary<NS, CNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)Seg::SMEM_IN),
                      "cudaFuncSetAttribute");
        VELO_CUDA_TRY(cudaFuncSetAttribute(k_gb_emit_rows<NS, CNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)Seg::SMEM),
                      "cudaFuncSetAttribute");
        if (dev >= 0 && dev < 64)
            done[dev] = 1;
    }
    const size_t np = s.n_rec;
    const int logN = ilog2_floor(np);
    VELO_CUDA_TRY(cudaMemsetAsync(s.rejected, 0, 8, st), "cudaMemsetAsync");
    k_gb_pack<NS><<<gb_grid(np), 256, 0, st>>>(in, n, np, s.r[0], s.r[1], s.r[2], s.rejected);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by pack launch");

    typename T::Rec::Cols rc;
    for (int i = 0; i < 1 + NS; i++) {
        rc.w[i] = s.r[i];
        rc.pad[i] = ~0ull;
    }
    rc.mask[0] = ~0ull;
    rc.mark_bit = 63;
    rc.mark_inv = 1;
    rc.mark_word = 0;
    std::vector<NetPass> passes;
    plan_sort(logN, GB_LT, GB_LMAX, passes);
    velo_status rc2 = launch_net12<typename T::Rec>(rc, NetGeom { np, logN, 0 }, passes, nullptr, st);
    if (rc2 != VELO_OK)
        return rc2;

    const int nts = (int)(np / SEG_TS);
    typename T::Grp::Cols gc;
    for (int i = 0; i < 1 + NS + CNT; i++) {
        gc.w[i] = s.g[i];
        gc.pad[i] = ~0ull;
    }
    gc.mask[0] = ~0ull;
    gc.mark_bit = 63;
    gc.mark_inv = 1;
    gc.mark_word = 0;
    k_gb_summary<NS, CNT><<<nts, SEG_THREADS, Seg::SMEM_IN, st>>>(rc, s.aggs, s.runs);
    k_gb_carries<NS, CNT><<<1, 1024, (NS + CNT) * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, nts, s.carry,
                                                                                 s.tail_prefix, s.n_groups);
    k_gb_emit_rows<NS, CNT><<<nts, SEG_THREADS, Seg::SMEM, st>>>(rc, nts, s.aggs, s.carry, gc);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by aggregation launch");

    const int ntc = (int)(np >> GB_LT);
    k_count_marks<typename T::Grp><<<ntc, 256, 0, st>>>(gc, np, GB_LT, s.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntc, s.prefix, s.n_grp_rows);
    passes.clear();
    plan_compact(logN, GB_LT, GB_LMAX, passes);
    rc2 = launch_net12<typename T::Grp>(gc, NetGeom { np, logN, 0 }, passes, s.prefix, st);
    if (rc2 != VELO_OK)
        return rc2;
    k_gb_out<NS, CNT><<<gb_grid(bound), 256, 0, st>>>(s.g[0], s.g[1], s.g[2], bound, in.key_type, out, s.n_groups,
                                                       s.rejected, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by output launch");
    return VELO_OK;
}

// BIGINT keys over their whole range: the same steps on wide records
static velo_status gb_run_wide(const GbScratch& s, const GbIn& in, int n_sums, int with_count, size_t n, size_t bound,
                               GbOut out, uint64_t* d_counts, cudaStream_t st)
{
    using T = GbTypesWide;
    using Seg = T::Seg;
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64 || !done[dev]) {
        VELO_CUDA_TRY(cudaFuncSetAttribute(k_gbw_summary, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)Seg::SMEM_IN),
                      "cudaFuncSetAttribute");
        VELO_CUDA_TRY(cudaFuncSetAttribute(k_gbw_emit_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)Seg::SMEM),
                      "cudaFuncSetAttribute");
        if (dev >= 0 && dev < 64)
            done[dev] = 1;
    }
    const size_t np = s.n_rec;
    const int logN = ilog2_floor(np);
    k_gb_pack_wide<<<gb_grid(np), 256, 0, st>>>(in, n_sums, n, np, s.r[0], s.r[1], s.r[2], s.r[3]);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by pack launch");
    T::Rec::Cols rc;
    for (int i = 0; i < 4; i++) {
        rc.w[i] = s.r[i];
        rc.pad[i] = ~0ull;
    }
    rc.pad[1] = 0; // network pads, if any, are rows left out
    rc.mask[0] = ~0ull;
    rc.mask[1] = ~0ull;
    rc.mark_bit = 0;
    rc.mark_inv = 0;
    rc.mark_word = 1;
    std::vector<NetPass> passes;
    plan_sort(logN, GB_LT, GB_LMAX, passes);
    velo_status rc2 = launch_net12<T::Rec>(rc, NetGeom { np, logN, 0 }, passes, nullptr, st);
    if (rc2 != VELO_OK)
        return rc2;
    const int nts = (int)(np / SEG_TS);
    T::Grp::Cols gc;
    for (int i = 0; i < 5; i++) {
        gc.w[i] = s.g[i];
        gc.pad[i] = ~0ull;
    }
    gc.mask[0] = ~0ull;
    gc.mark_bit = 63;
    gc.mark_inv = 1;
    gc.mark_word = 1;
    k_gbw_summary<<<nts, SEG_THREADS, Seg::SMEM_IN, st>>>(rc, s.aggs, s.runs);
    k_gbw_carries<<<1, 1024, 3 * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, nts, s.carry, s.tail_prefix,
                                                                s.n_groups);
    k_gbw_emit_rows<<<nts, SEG_THREADS, Seg::SMEM, st>>>(rc, nts, s.aggs, s.carry, gc);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by aggregation launch");
    const int ntc = (int)(np >> GB_LT);
    k_count_marks<T::Grp><<<ntc, 256, 0, st>>>(gc, np, GB_LT, s.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntc, s.prefix, s.n_grp_rows);
    passes.clear();
    plan_compact(logN, GB_LT, GB_LMAX, passes);
    rc2 = launch_net12<T::Grp>(gc, NetGeom { np, logN, 0 }, passes, s.prefix, st);
    if (rc2 != VELO_OK)
        return rc2;
    GbwWords gw;
    for (int i = 0; i < 5; i++)
        gw.g[i] = s.g[i];
    k_gbw_out<<<gb_grid(bound), 256, 0, st>>>(gw, bound, n_sums, with_count, out, s.n_groups, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by output launch");
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_ogroupby_scratch_bytes(size_t n) { return gb_layout(nullptr, n).bytes; }

extern "C" velo_status velo_ogroupby(const void* d_keys, uint32_t key_type, const int64_t* const* d_sums,
                                     uint32_t n_sums, uint32_t with_count, const uint8_t* d_mask, size_t n,
                                     size_t group_bound, int64_t* d_out_keys, int64_t* const* d_out_sums,
                                     int64_t* d_out_counts, uint64_t* d_counts, void* d_scratch, size_t scratch_bytes,
                                     void* stream)
{
    const uint32_t v = n_sums + (with_count ? 1u : 0u);
    if (v < 1 || v > 2)
        return einval("velo_ogroupby: one or two aggregates per call (n_sums + with_count)");
    if (key_type != VELO_INTEGER && key_type != VELO_BIGINT)
        return einval("velo_ogroupby: key_type must be VELO_INTEGER or VELO_BIGINT");
    if (n == 0 || group_bound == 0 || group_bound > n)
        return einval("velo_ogroupby: need 1 <= group_bound <= n");
    if (next_pow2(n) > ((size_t)1 << MAX_LOGN))
        return einval("velo_ogroupby: n above 2^31");
    if (!d_keys || !d_out_keys || !d_counts || (with_count && !d_out_counts) || (n_sums && (!d_sums || !d_out_sums)))
        return einval("velo_ogroupby: null argument");
    for (uint32_t i = 0; i < n_sums; i++)
        if (!d_sums[i] || !d_out_sums[i])
            return einval("velo_ogroupby: null sum column");
    GbScratch s = gb_layout(static_cast<char*>(d_scratch), n);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ogroupby: scratch must hold velo_ogroupby_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    GbIn in {};
    in.keys = d_keys;
    in.mask = d_mask;
    in.key_type = key_type;
    GbOut out {};
    out.keys = d_out_keys;
    out.counts = d_out_counts;
    for (uint32_t i = 0; i < n_sums; i++) {
        in.sums[i] = d_sums[i];
        out.sums[i] = d_out_sums[i];
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (key_type == VELO_BIGINT)
        return gb_run_wide(s, in, (int)n_sums, with_count ? 1 : 0, n, group_bound, out, d_counts, st);
    if (with_count && n_sums == 0)
        return gb_run<0, 1>(s, in, n, group_bound, out, d_counts, st);
    if (with_count && n_sums == 1)
        return gb_run<1, 1>(s, in, n, group_bound, out, d_counts, st);
    if (n_sums == 1)
        return gb_run<1, 0>(s, in, n, group_bound, out, d_counts, st);
    return gb_run<2, 0>(s, in, n, group_bound, out, d_counts, st);
}
