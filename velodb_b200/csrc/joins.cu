// Oblivious many-to-many equi-join (velo_ojoin_mn): every pair (build row,
// probe row) with equal keys, both rows valid, padded to a public bound of
// max_pairs output rows.
//
// The reference's sort-merge join (include/cuda/sort_merge_join.cuh:63-199,
// src/operator/sort_merge_join_operator.cpp:27-257) merges the two sorted
// sides block by block and writes the cross product of every run of equal
// keys; its loops, binary searches and atomics depend on the data.  Here every
// step is a network pass or a streaming pass over public sizes:
//
//   1. union   U = next_pow2(build_n + probe_n) records
//              w0 = key (order-preserving), w1 = [63] row left out | [62] tag
//              (0 build, 1 probe) | [61] valid build | [31:0] row id
//   2. sort    bitonic network on (w0, w1): each key's valid build rows in row
//              id order, then its valid probe rows, then the rows left out
//   3. scan 1  per row: P = valid build rows before it, c = valid build rows of
//              its key before it; for a valid probe row c is its number of
//              partners and P - c the position of its key's first build row in
//              the key-ordered build list
//   4. scan 2  dest = exclusive prefix of c over the valid probe rows: the
//              first output slot of each probe row; the total is the pair count
//   5. expand  E = next_pow2(U + max_pairs) records: one per probe row with
//              partners (position dest), one per output slot s (position s);
//              sort on (position, slot flag); a forward fill hands every slot
//              the last probe row at or before it; slot s < dest + c takes
//              probe row id and build position P - c + (s - dest); an
//              ORCompact brings the slot records back in slot order
//   6. build   ORCompact of the sorted union on the valid-build flag gives the
//              key-ordered build row ids; an oblivious gather (union sort,
//              fill, sort back) reads the build row id of every slot
//
// Output row s < min(pairs, max_pairs) holds the s-th pair in (key, probe row
// id, build row id) order; the rest hold -1.  Every launch, address and
// branch depends only on build_n, probe_n and max_pairs.
#include <algorithm>
#include <cmath>

#include "union.cuh"

namespace velo {

// exclusive scan of run summaries of tiles: one CTA of 1024 threads, rounds of
// 1024 consecutive tiles chained through the running total
__global__ void __launch_bounds__(1024) k_run_scan(const RunSum* tiles, int ntiles, RunSum* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_run_scan"));
    __shared__ RunSum sm[1024];
    RunSum run {};
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int t = base + (int)threadIdx.x;
        RunSum x {};
        if (t < ntiles) {
            VELO_TRACE_AT(TS_FILL, tiles + t);
            x = tiles[t];
        }
        RunSum total;
        const RunSum ex = run_block_scan_excl(x, sm, &total);
        if (t < ntiles)
            carry[t] = run_combine(run, ex);
        run = run_combine(run, total);
    }
}


constexpr uint64_t MN_OUT = 1ull << 63, MN_TAG = 1ull << 62, MN_VB = 1ull << 61;
constexpr uint64_t MN_ROWID = 0xFFFFFFFFull;
constexpr int MN_TS = 2048, MN_THREADS = 256, MN_RPT = MN_TS / MN_THREADS;

__device__ __forceinline__ bool mn_valid_build(uint64_t w1) { return (w1 & (MN_OUT | MN_TAG)) == 0; }
__device__ __forceinline__ bool mn_valid_probe(uint64_t w1) { return (w1 & (MN_OUT | MN_TAG)) == MN_TAG; }

__global__ void k_mn_pack(const void* bk, const uint8_t* bm, size_t bn, const void* pk, const uint8_t* pm, size_t pn,
                          int key64, size_t rows, uint64_t* w0, uint64_t* w1, uint64_t* w2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_pack"));
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, rows);
         g += (size_t)gridDim.x * blockDim.x) {
        uint64_t a = ~0ull, b = ~0ull;
        if (g < bn + pn) {
            const bool build = g < bn;
            const size_t j = build ? g : g - bn;
            const void* keys = build ? bk : pk;
            const uint8_t* mask = build ? bm : pm;
            a = key64 ? ((uint64_t) static_cast<const int64_t*>(keys)[j] ^ 0x8000000000000000ull)
                      : (uint64_t)((uint32_t) static_cast<const int32_t*>(keys)[j] ^ 0x80000000u);
            const bool valid = mask == nullptr || mask[j] != 0;
            b = (valid ? 0ull : MN_OUT) | (build ? 0ull : MN_TAG) | ((valid & build) ? MN_VB : 0ull) | (uint64_t)j;
        }
        VELO_TRACE_AT(TS_ROW_STORE, w0 + g);
        w0[g] = a;
        w1[g] = b;
        w2[g] = 0;
    }
}

// ---- scan 1: segmented count of valid build rows over key runs ---------------

__global__ void __launch_bounds__(MN_THREADS) k_mn_sum1(const uint64_t* w0, const uint64_t* w1, RunSum* tiles)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_sum1"));
    __shared__ RunSum sm[MN_THREADS];
    const size_t base = (size_t)blockIdx.x * MN_TS + (size_t)threadIdx.x * MN_RPT;
    RunSum s {};
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        s = run_combine(s, run_row(w0[base + r], mn_valid_build(w1[base + r]) ? 1ull : 0ull));
    }
    RunSum total;
    run_block_scan_excl(s, sm, &total);
    if (threadIdx.x == 0) {
        VELO_TRACE_AT(TS_FILL, tiles + blockIdx.x);
        tiles[blockIdx.x] = total;
    }
}

// Per row: c (valid build rows of its key before it) and P - c for valid probe
// rows, stored as w2 = (P - c) << 32 | c; the tile-local exclusive prefix of c
// over valid probe rows replaces w0 (the key is no longer needed); the tile's
// total of c goes to csum.
__global__ void __launch_bounds__(MN_THREADS) k_mn_apply1(uint64_t* w0, uint64_t* w1, uint64_t* w2,
                                                          const RunSum* carry, uint64_t* csum)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_apply1"));
    __shared__ RunSum sm[MN_THREADS];
    __shared__ uint64_t s64[MN_THREADS];
    const size_t base = (size_t)blockIdx.x * MN_TS + (size_t)threadIdx.x * MN_RPT;
    uint64_t k[MN_RPT], b[MN_RPT];
    RunSum s {};
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        k[r] = w0[base + r];
        b[r] = w1[base + r];
        s = run_combine(s, run_row(k[r], mn_valid_build(b[r]) ? 1ull : 0ull));
    }
    RunSum total;
    RunSum run = run_combine(carry[blockIdx.x], run_block_scan_excl(s, sm, &total));
    uint64_t cs[MN_RPT], c_thread = 0;
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        // run covers the rows before row r: P = run.nb, and the builds of
        // this row's key before it are run.tail_nb when run ends in this key
        const uint64_t P = run.has ? run.nb : 0ull;
        const uint64_t c = (run.has && run.last_key == k[r]) ? run.tail_nb : 0ull;
        const bool probe = mn_valid_probe(b[r]);
        cs[r] = probe ? c : 0ull;
        c_thread += cs[r];
        w2[base + r] = probe ? (((P - c) << 32) | c) : 0ull;
        run = run_combine(run, run_row(k[r], mn_valid_build(b[r]) ? 1ull : 0ull));
    }
    // tile-local exclusive prefix of c over the threads (then within each)
    uint64_t x = c_thread;
    const int t = threadIdx.x;
    for (int off = 1; off < MN_THREADS; off <<= 1) {
        __syncthreads();
        s64[t] = x;
        __syncthreads();
        if (t >= off)
            x += s64[t - off];
    }
    uint64_t pre = x - c_thread;
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        w0[base + r] = pre;
        pre += cs[r];
    }
    if (t == MN_THREADS - 1)
        csum[blockIdx.x] = x;
}

// exclusive scan of the tile totals of c (one CTA), and the pair count
__global__ void __launch_bounds__(1024) k_mn_scan2(const uint64_t* csum, int ntiles, uint64_t* cbase, uint64_t* pairs)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_scan2"));
    __shared__ uint64_t sm[1024];
    uint64_t run = 0;
    const int t = threadIdx.x;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int i = base + t;
        const uint64_t v = i < ntiles ? csum[i] : 0ull;
        uint64_t x = v;
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            __syncthreads();
            sm[t] = x;
            __syncthreads();
            if (t >= off)
                x += sm[t - off];
        }
        if (i < ntiles)
            cbase[i] = run + x - v;
        __syncthreads();
        sm[t] = x;
        __syncthreads();
        run += sm[blockDim.x - 1];
        __syncthreads();
    }
    if (t == 0)
        *pairs = run;
}

// ---- expansion ----------------------------------------------------------------

// expansion records: probe row  e0 = dest << 1, e1 = probe row id << 32 | c,
//                                e2 = build position of its key's first row
//                    slot s      e0 = s << 1 | 1, e1 = 0, e2 = s
//                    other rows  all ones
__global__ void k_mn_expand_pack(const uint64_t* w0, const uint64_t* w1, const uint64_t* w2, size_t U,
                                 const uint64_t* cbase, size_t max_pairs, size_t E, uint64_t* e0, uint64_t* e1,
                                 uint64_t* e2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_expand_pack"));
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, E);
         g += (size_t)gridDim.x * blockDim.x) {
        uint64_t a = ~0ull, b = ~0ull, c = ~0ull;
        if (g < U) {
            VELO_TRACE_AT(TS_FILL, w1 + g);
            const uint64_t x1 = w1[g], x2 = w2[g];
            const uint64_t dest = cbase[g / MN_TS] + w0[g];
            const uint64_t cnt = x2 & 0xFFFFFFFFull;
            const bool take = mn_valid_probe(x1) & (cnt != 0) & (dest < max_pairs);
            a = take ? (dest << 1) : ~0ull;
            b = take ? (((x1 & MN_ROWID) << 32) | cnt) : ~0ull;
            c = take ? (x2 >> 32) : ~0ull;
        } else if (g - U < max_pairs) {
            const uint64_t s = g - U;
            a = (s << 1) | 1ull;
            b = 0;
            c = s;
        }
        VELO_TRACE_AT(TS_ROW_STORE, e0 + g);
        e0[g] = a;
        e1[g] = b;
        e2[g] = c;
    }
}

// forward fill: every slot record takes the last probe record at or before it
struct MnExpandFill {
    __device__ __forceinline__ static bool is_probe(uint64_t a) { return a != ~0ull && (a & 1ull) == 0; }
    __device__ __forceinline__ static bool is_slot(uint64_t a) { return a != ~0ull && (a & 1ull) == 1; }
    __device__ __forceinline__ static FillCarry src(uint64_t a, uint64_t b, uint64_t c)
    {
        // key = build position << 32 | dest, val = probe row id << 32 | c
        const bool p = is_probe(a);
        return FillCarry { ((c & 0xFFFFFFFFull) << 32) | ((a >> 1) & 0xFFFFFFFFull), b, p ? 1u : 0u, 1u };
    }
    __device__ __forceinline__ static bool dup(uint64_t, uint64_t, uint64_t, const FillCarry&) { return false; }
    __device__ __forceinline__ static void apply(uint64_t& a, uint64_t& b, uint64_t& c, const FillCarry& last)
    {
        const bool slot = is_slot(a);
        const uint64_t s = a >> 1;
        const uint64_t dest = last.key & 0xFFFFFFFFull, lstart = last.key >> 32;
        const uint64_t cnt = last.val & 0xFFFFFFFFull, rowid = last.val >> 32;
        const uint64_t t = s - dest;
        const bool hit = slot & (last.has != 0) & (s >= dest) & (t < cnt);
        b = hit ? rowid : ~0ull;
        c = hit ? (lstart + t) : ~0ull;
        // only slot records stay marked (bit 0) for the compaction
        a = slot ? a : 0ull;
    }
};

// slot s: probe row id, and the build position to gather (0 for an empty slot)
__global__ void k_mn_slots_out(const uint64_t* e1, const uint64_t* e2, size_t max_pairs, int64_t* out_probe,
                               uint32_t* lpos)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_slots_out"));
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(s, max_pairs);
         s += (size_t)gridDim.x * blockDim.x) {
        VELO_TRACE_AT(TS_ROW_LOAD, e1 + s);
        const uint64_t b = e1[s], c = e2[s];
        const bool hit = b != ~0ull;
        out_probe[s] = hit ? (int64_t)b : -1;
        lpos[s] = hit ? (uint32_t)c : 0u;
    }
}

// the key-ordered build row ids (the first valid-build rows after the
// compaction of the sorted union)
__global__ void k_mn_build_table(const uint64_t* w1, size_t n, uint64_t* table)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_build_table"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n);
         i += (size_t)gridDim.x * blockDim.x) {
        VELO_TRACE_AT(TS_ROW_LOAD, w1 + i);
        table[i] = w1[i] & MN_ROWID;
    }
}

__global__ void k_mn_out(const uint64_t* gathered, const int64_t* out_probe, size_t max_pairs, int64_t* out_build,
                         const uint64_t* pairs, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mn_out"));
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(s, max_pairs);
         s += (size_t)gridDim.x * blockDim.x) {
        VELO_TRACE_AT(TS_ROW_LOAD, gathered + s);
        out_build[s] = out_probe[s] >= 0 ? (int64_t)gathered[s] : -1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint64_t p = *pairs;
        d_counts[0] = p;
        d_counts[1] = p > max_pairs ? 1ull : 0ull;
    }
}

// ---- scratch ------------------------------------------------------------------

struct MnScratch {
    size_t U, E;
    UnionScratch u;    // sorted union
    UnionScratch e;    // expansion (its area is reused by the gather)
    size_t e_off, e_bytes;
    RunSum* tiles;
    RunSum* carry;
    uint64_t* csum;
    uint64_t* cbase;
    uint64_t* pairs;
    uint32_t* lpos;
    uint64_t* gathered;
    uint64_t* table;
    size_t bytes;
};

static size_t mn_gather_bytes(size_t build_n, size_t max_pairs)
{
    return union_layout(nullptr, union_rows(build_n + max_pairs)).bytes;
}

static MnScratch mn_layout(char* base, size_t build_n, size_t probe_n, size_t max_pairs)
{
    MnScratch s {};
    s.U = union_rows(build_n + probe_n);
    s.E = union_rows(s.U + max_pairs);
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += align_up(b ? b : 1, 256);
        return p;
    };
    const size_t ub = union_layout(nullptr, s.U).bytes;
    s.u = union_layout(static_cast<char*>(take(ub)), s.U);
    const size_t eb = std::max(union_layout(nullptr, s.E).bytes, mn_gather_bytes(build_n, max_pairs));
    s.e_off = off;
    s.e_bytes = eb;
    s.e = union_layout(static_cast<char*>(take(eb)), s.E);
    const size_t nt = s.U / MN_TS;
    s.tiles = reinterpret_cast<RunSum*>(take(nt * sizeof(RunSum)));
    s.carry = reinterpret_cast<RunSum*>(take(nt * sizeof(RunSum)));
    s.csum = reinterpret_cast<uint64_t*>(take(nt * 8));
    s.cbase = reinterpret_cast<uint64_t*>(take(nt * 8));
    s.pairs = reinterpret_cast<uint64_t*>(take(8));
    s.lpos = reinterpret_cast<uint32_t*>(take(max_pairs * 4));
    s.gathered = reinterpret_cast<uint64_t*>(take(max_pairs * 8));
    s.table = reinterpret_cast<uint64_t*>(take((build_n ? build_n : 1) * 8));
    s.bytes = off;
    if (!base) {
        s.u = union_layout(nullptr, s.U);
        s.e = union_layout(nullptr, s.E);
    }
    return s;
}

static unsigned mn_grid(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_ojoin_mn_scratch_bytes(size_t build_n, size_t probe_n, size_t max_pairs)
{
    return mn_layout(nullptr, build_n, probe_n, max_pairs ? max_pairs : 1).bytes;
}

extern "C" velo_status velo_ojoin_mn(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                                     const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n,
                                     uint32_t key_type, size_t max_pairs, int64_t* d_out_build_rowid,
                                     int64_t* d_out_probe_rowid, uint64_t* d_counts, void* d_scratch,
                                     size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_counts)
        return einval("velo_ojoin_mn: null counts");
    if (key_type != VELO_INTEGER && key_type != VELO_BIGINT)
        return einval("velo_ojoin_mn: join keys must be INTEGER or BIGINT");
    if (max_pairs == 0)
        return einval("velo_ojoin_mn: max_pairs must be at least 1");
    if (!d_out_build_rowid || !d_out_probe_rowid)
        return einval("velo_ojoin_mn: null output");
    if (build_n >= 0x80000000ull || probe_n >= 0x80000000ull || max_pairs >= 0x80000000ull)
        return einval("velo_ojoin_mn: sizes must be below 2^31");
    if (probe_n == 0 || build_n == 0) {
        VELO_CUDA_TRY(cudaMemsetAsync(d_counts, 0, 16, st), "cudaMemsetAsync");
        VELO_CUDA_TRY(cudaMemsetAsync(d_out_build_rowid, 0xFF, max_pairs * 8, st), "cudaMemsetAsync");
        VELO_CUDA_TRY(cudaMemsetAsync(d_out_probe_rowid, 0xFF, max_pairs * 8, st), "cudaMemsetAsync");
        return VELO_OK;
    }
    if (!d_build_keys || !d_probe_keys)
        return einval("velo_ojoin_mn: null keys");
    MnScratch s = mn_layout(static_cast<char*>(d_scratch), build_n, probe_n, max_pairs);
    if (ilog2_floor(s.E) > MAX_LOGN)
        return einval("velo_ojoin_mn: build_n + probe_n + max_pairs too large");
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ojoin_mn: scratch must hold velo_ojoin_mn_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    const size_t U = s.U, E = s.E;
    const int logU = ilog2_floor(U), logE = ilog2_floor(E);
    uint64_t* const* w = s.u.w;

    // 1-2. union and sort on (key, row flags)
    k_mn_pack<<<mn_grid(U), 256, 0, st>>>(d_build_keys, d_build_mask, build_n, d_probe_keys, d_probe_mask, probe_n,
                                          key_type == VELO_BIGINT, U, w[0], w[1], w[2]);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn pack launch");
    Rec3K2::Cols uc;
    for (int i = 0; i < 3; i++) {
        uc.w[i] = w[i];
        uc.pad[i] = ~0ull;
    }
    uc.mask[0] = ~0ull;
    uc.mask[1] = ~0ull;
    uc.mark_word = 1;
    uc.mark_bit = 61; // the valid-build flag, for step 6
    uc.mark_inv = 0;
    std::vector<NetPass> passes;
    plan_sort(logU, OP_LT, OP_LMAX, passes);
    velo_status rc = launch_net12<Rec3K2>(uc, NetGeom { U, logU, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;

    // 3-4. the two scans
    const int nt = (int)(U / MN_TS);
    k_mn_sum1<<<nt, MN_THREADS, 0, st>>>(w[0], w[1], s.tiles);
    k_run_scan<<<1, 1024, 0, st>>>(s.tiles, nt, s.carry);
    k_mn_apply1<<<nt, MN_THREADS, 0, st>>>(w[0], w[1], w[2], s.carry, s.csum);
    k_mn_scan2<<<1, 1024, 0, st>>>(s.csum, nt, s.cbase, s.pairs);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn scan launch");

    // 5. expansion into max_pairs slots
    uint64_t* const* e = s.e.w;
    k_mn_expand_pack<<<mn_grid(E), 256, 0, st>>>(w[0], w[1], w[2], U, s.cbase, max_pairs, E, e[0], e[1], e[2]);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn expand launch");
    Rec3::Cols ec;
    for (int i = 0; i < 3; i++) {
        ec.w[i] = e[i];
        ec.pad[i] = ~0ull;
    }
    ec.mask[0] = ~0ull;
    ec.mark_word = 0;
    ec.mark_bit = 0; // slot records
    ec.mark_inv = 0;
    passes.clear();
    plan_sort(logE, OP_LT, OP_LMAX, passes);
    rc = launch_net12<Rec3>(ec, NetGeom { E, logE, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    rc = run_fill<MnExpandFill>(e[0], e[1], e[2], E, s.e.tl, s.e.carry, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    const int nce = (int)(E >> OP_LT);
    k_count_marks<Rec3><<<nce, 256, 0, st>>>(ec, E, OP_LT, s.e.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.e.counts, nce, s.e.prefix, s.e.n_marked);
    passes.clear();
    plan_compact(logE, OP_LT, OP_LMAX, passes);
    rc = launch_net12<Rec3>(ec, NetGeom { E, logE, 0 }, passes, s.e.prefix, st);
    if (rc != VELO_OK)
        return rc;
    k_mn_slots_out<<<mn_grid(max_pairs), 256, 0, st>>>(e[1], e[2], max_pairs, d_out_probe_rowid, s.lpos);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn slots launch");

    // 6. key-ordered build row ids, and the gather of each slot's build row
    const int ncu = (int)(U >> OP_LT);
    k_count_marks<Rec3K2><<<ncu, 256, 0, st>>>(uc, U, OP_LT, s.u.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.u.counts, ncu, s.u.prefix, s.u.n_marked);
    passes.clear();
    plan_compact(logU, OP_LT, OP_LMAX, passes);
    rc = launch_net12<Rec3K2>(uc, NetGeom { U, logU, 0 }, passes, s.u.prefix, st);
    if (rc != VELO_OK)
        return rc;
    k_mn_build_table<<<mn_grid(build_n), 256, 0, st>>>(w[1], build_n, s.table);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn table launch");
    rc = velo_ogather_u64(s.table, build_n, s.lpos, max_pairs, s.gathered, static_cast<char*>(d_scratch) + s.e_off,
                          s.e_bytes, stream);
    if (rc != VELO_OK)
        return rc;
    k_mn_out<<<mn_grid(max_pairs), 256, 0, st>>>(s.gathered, d_out_probe_rowid, max_pairs, d_out_build_rowid, s.pairs,
                                                 d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin_mn out launch");
    return VELO_OK;
}

// ===========================================================================
// Oblivious bin-padded hash join (velo_ohash_join)
//
// The reference's hash join (include/cuda/hash_join.cuh:28-254,
// src/operator/hash_join_operator.cpp:88-393) chains build rows into a hash
// table and walks the chains for every probe row; its addresses follow the
// keys.  Here both sides are hashed into B bins by a keyed Philox4x32-10 hash
// and every bin is padded to a public capacity (C_b build slots, C_p probe
// slots, set from the public sizes), so a bin's occupancy never shows:
//
//   1. union   R = next_pow2(build_n + probe_n + B (C_b + C_p)) records
//              w0 = [63] not kept | bin << 33 | side << 32 | dummy << 31
//                   | row id (dummy: slot index), w1 = key; rows left out
//              by their mask take bin B (no bin); every bin also gets C_b
//              build dummies and C_p probe dummies
//   2. sort    bitonic network on w0: each (bin, side) group holds its real
//              rows in row id order, then its dummies
//   3. rank    a run-count scan gives each row its rank in its group; the
//              first C rows of every group are kept (real rows first), real
//              rows past the capacity are counted as overflow
//   4. place   ORCompact of the kept rows: slot b (C_b + C_p) + i is bin b's
//              i-th build slot, then its probe slots
//   5. bins    one CTA per bin holds the C_b build slots in shared memory and
//              compares every probe slot with every build slot, reading the
//              build slots in the same order for every bin (a broadcast
//              read, no data-dependent address); a probe slot with two or
//              more partners counts a repeated build key
//   6. output  ORCompact of the joined probe slots; the first `pairs` rows
//              are (build row id, probe row id) in (bin, probe row id) order,
//              the rest up to probe_n are -1
//
// Every launch, address and branch depends only on build_n, probe_n and the
// hash seed.  Overflow (a bin holding more rows than its capacity) and a
// repeated build key are reported in d_counts; the caller then joins with the
// sort-merge join (velo_ojoin_mn), which has no such limit.
// ===========================================================================

namespace velo {

constexpr uint64_t HJ_DROP = 1ull << 63, HJ_SIDE = 1ull << 32, HJ_DUMMY = 1ull << 31;
constexpr uint64_t HJ_ID = (1ull << 31) - 1;
constexpr int HJ_THREADS = 512;

struct HjGeom {
    uint32_t B, log_b, cb, cp; // bins, log2 bins, build / probe slots per bin
    size_t rows;               // padded union rows
    size_t slots;              // B (cb + cp)
    size_t probe_slots;        // B cp
    size_t out_rows;           // padded probe slot records (>= B cp)
};

static uint32_t hj_cap(size_t mean, double sigmas)
{
    const double c = (double)mean + sigmas * std::sqrt((double)mean) + 16.0;
    return (uint32_t)((((uint64_t)std::ceil(c)) + 31) / 32 * 32);
}

// mean build rows per bin in [1024, 2048) (a single bin below); the build
// capacity allows 8 standard deviations of a Poisson count, the probe side
// 16, because foreign keys repeat and their bin counts spread wider
static HjGeom hj_geometry(size_t build_n, size_t probe_n)
{
    HjGeom g {};
    uint32_t B = 1, lb = 0;
    while ((size_t)B * 2 * 1024 <= build_n && lb < 20) {
        B *= 2;
        lb++;
    }
    g.B = B;
    g.log_b = lb;
    g.cb = hj_cap((build_n + B - 1) / B, 8.0);
    g.cp = hj_cap((probe_n + B - 1) / B, 16.0);
    g.slots = (size_t)B * (g.cb + g.cp);
    g.probe_slots = (size_t)B * g.cp;
    g.rows = union_rows(build_n + probe_n + g.slots);
    g.out_rows = union_rows(g.probe_slots);
    return g;
}

__device__ __forceinline__ uint64_t hj_key(const void* keys, size_t j, int key64)
{
    return key64 ? ((uint64_t) static_cast<const int64_t*>(keys)[j] ^ 0x8000000000000000ull)
                 : (uint64_t)((uint32_t) static_cast<const int32_t*>(keys)[j] ^ 0x80000000u);
}

__global__ void k_hj_pack(const void* bk, const uint8_t* bm, size_t bn, const void* pk, const uint8_t* pm, size_t pn,
                          int key64, HjGeom g, uint64_t seed, uint64_t* w0, uint64_t* w1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_hj_pack"));
    const size_t real = bn + pn, bdum = (size_t)g.B * g.cb;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, g.rows);
         i += (size_t)gridDim.x * blockDim.x) {
        uint64_t a = ~0ull, b = ~0ull;
        if (i < real) {
            const bool build = i < bn;
            const size_t j = build ? i : i - bn;
            const uint64_t key = hj_key(build ? bk : pk, j, key64);
            const uint8_t* mask = build ? bm : pm;
            const bool valid = mask == nullptr || mask[j] != 0;
            const uint64_t bin = valid ? (philox_u64(key, 0x4A4F494Eull, seed) & (g.B - 1ull)) : (uint64_t)g.B;
            a = (bin << 33) | (build ? 0ull : HJ_SIDE) | (uint64_t)j;
            b = key;
        } else if (i < real + g.slots) {
            const size_t d = i - real;
            const bool build = d < bdum;
            const size_t e = build ? d : d - bdum;
            const uint32_t cap = build ? g.cb : g.cp;
            const uint64_t bin = e / cap, slot = e - bin * cap;
            a = (bin << 33) | (build ? 0ull : HJ_SIDE) | HJ_DUMMY | slot;
            b = 0;
        }
        VELO_TRACE_AT(TS_ROW_STORE, w0 + i);
        w0[i] = a;
        w1[i] = b;
    }
}

// group key of a placement record: (bin, side); pads have their own
__device__ __forceinline__ uint64_t hj_group(uint64_t w0) { return (w0 & ~HJ_DROP) >> 32; }

__global__ void __launch_bounds__(MN_THREADS) k_hj_sum(const uint64_t* w0, RunSum* tiles)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_hj_sum"));
    __shared__ RunSum sm[MN_THREADS];
    const size_t base = (size_t)blockIdx.x * MN_TS + (size_t)threadIdx.x * MN_RPT;
    RunSum s {};
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        s = run_combine(s, run_row(hj_group(w0[base + r]), 1ull));
    }
    RunSum total;
    run_block_scan_excl(s, sm, &total);
    if (threadIdx.x == 0) {
        VELO_TRACE_AT(TS_FILL, tiles + blockIdx.x);
        tiles[blockIdx.x] = total;
    }
}

// rank in the (bin, side) group: keep the first C rows of every bin's group,
// count real rows past the capacity (one counter update per CTA)
__global__ void __launch_bounds__(MN_THREADS) k_hj_rank(uint64_t* w0, const RunSum* carry, uint32_t B, uint32_t cb,
                                                        uint32_t cp, unsigned long long* overflow)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_hj_rank"));
    __shared__ RunSum sm[MN_THREADS];
    __shared__ uint32_t tmp[33];
    const size_t base = (size_t)blockIdx.x * MN_TS + (size_t)threadIdx.x * MN_RPT;
    uint64_t a[MN_RPT];
    RunSum s {};
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        a[r] = w0[base + r];
        s = run_combine(s, run_row(hj_group(a[r]), 1ull));
    }
    RunSum total;
    RunSum run = run_combine(carry[blockIdx.x], run_block_scan_excl(s, sm, &total));
    uint32_t over = 0;
#pragma unroll
    for (int r = 0; r < MN_RPT; r++) {
        const uint64_t grp = hj_group(a[r]);
        const uint64_t rank = (run.has && run.last_key == grp) ? run.tail_nb : 0ull;
        const uint64_t bin = grp >> 1;
        const uint32_t cap = (grp & 1ull) ? cp : cb;
        const bool pad = a[r] == ~0ull;
        const bool keep = !pad & (bin < B) & (rank < cap);
        over += (!pad & (bin < B) & ((a[r] & HJ_DUMMY) == 0) & (rank >= cap)) ? 1u : 0u;
        VELO_TRACE_AT(TS_FILL, w0 + base + r);
        w0[base + r] = keep ? (a[r] & ~HJ_DROP) : (a[r] | HJ_DROP);
        run = run_combine(run, run_row(grp, 1ull));
    }
    uint32_t t;
    block_exclusive_scan(over, tmp, &t);
    if (threadIdx.x == 0 && t)
        atomicAdd(overflow, (unsigned long long)t);
}

// one CTA per bin: every probe slot against every build slot of the bin
// probe slot record: o0 = [63] not joined | probe row id, o1 = build row id
__global__ void __launch_bounds__(HJ_THREADS) k_hj_bins(const uint64_t* w0, const uint64_t* w1, HjGeom g,
                                                        size_t out_rows, uint64_t* o0, uint64_t* o1,
                                                        unsigned long long* dups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_hj_bins"));
    extern __shared__ __align__(16) char smem[];
    uint64_t* bkey = reinterpret_cast<uint64_t*>(smem);
    uint64_t* brow = bkey + g.cb; // row id, or ~0 for a dummy
    __shared__ uint32_t tmp[33];
    const size_t bin = blockIdx.x;
    const size_t base = bin * (size_t)(g.cb + g.cp);
    for (uint32_t i = threadIdx.x; i < g.cb; i += blockDim.x) {
        VELO_TRACE_AT(TS_ROW_LOAD, w0 + base + i);
        const uint64_t a = w0[base + i];
        bkey[i] = w1[base + i];
        brow[i] = (a & HJ_DUMMY) ? ~0ull : (a & HJ_ID);
    }
    __syncthreads();
    uint32_t dup = 0;
    for (uint32_t p0 = threadIdx.x; p0 < g.cp; p0 += 4 * blockDim.x) {
        uint64_t pkey[4], prow[4], hit[4];
        uint32_t cnt[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t p = p0 + q * blockDim.x;
            const bool in = p < g.cp;
            const size_t gi = base + g.cb + (in ? p : 0);
            VELO_TRACE_AT(TS_ROW_LOAD, w0 + gi);
            const uint64_t a = w0[gi];
            pkey[q] = w1[gi];
            prow[q] = (!in || (a & HJ_DUMMY)) ? ~0ull : (a & HJ_ID);
            hit[q] = ~0ull;
            cnt[q] = 0;
        }
        for (uint32_t j = 0; j < g.cb; j++) {
            const uint64_t k = bkey[j], r = brow[j];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const bool eq = (k == pkey[q]) & (r != ~0ull);
                hit[q] = eq ? r : hit[q];
                cnt[q] += eq ? 1u : 0u;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t p = p0 + q * blockDim.x;
            const bool joined = (prow[q] != ~0ull) & (cnt[q] != 0);
            dup += (prow[q] != ~0ull && cnt[q] > 1) ? 1u : 0u;
            if (p < g.cp) {
                const size_t o = bin * (size_t)g.cp + p;
                VELO_TRACE_AT(TS_ROW_STORE, o0 + o);
                o0[o] = joined ? (prow[q] & HJ_ID) : (HJ_DROP | (prow[q] & HJ_ID));
                o1[o] = joined ? hit[q] : ~0ull;
            }
        }
    }
    uint32_t t;
    block_exclusive_scan(dup, tmp, &t);
    if (threadIdx.x == 0 && t)
        atomicAdd(dups, (unsigned long long)t);
    // the pad records after the last bin's slots
    if (blockIdx.x == 0)
        for (size_t i = g.probe_slots + threadIdx.x; i < out_rows; i += blockDim.x) {
            o0[i] = ~0ull;
            o1[i] = ~0ull;
        }
}

__global__ void k_hj_out(const uint64_t* o0, const uint64_t* o1, size_t pn, const uint64_t* pairs,
                         const unsigned long long* dups, const unsigned long long* overflow, int64_t* ob, int64_t* op,
                         uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_hj_out"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, pn);
         i += (size_t)gridDim.x * blockDim.x) {
        VELO_TRACE_AT(TS_ROW_LOAD, o0 + i);
        const uint64_t a = o0[i];
        const bool j = (a & HJ_DROP) == 0;
        ob[i] = j ? (int64_t)o1[i] : -1;
        op[i] = j ? (int64_t)(a & HJ_ID) : -1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d_counts[0] = *pairs;
        d_counts[1] = *dups;
        d_counts[2] = *overflow;
    }
}

struct HjScratch {
    HjGeom g;
    uint64_t* w[2];
    uint64_t* o[2];
    RunSum* tiles;
    RunSum* carry;
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* n_marked;
    uint32_t* ocounts;
    uint32_t* oprefix;
    uint64_t* pairs;
    unsigned long long* stat; // [0] repeated build keys, [1] overflow
    size_t bytes;
};

static HjScratch hj_layout(char* base, size_t build_n, size_t probe_n)
{
    HjScratch s {};
    s.g = hj_geometry(build_n, probe_n);
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = base ? base + off : nullptr;
        off += align_up(b ? b : 1, 256);
        return p;
    };
    for (int i = 0; i < 2; i++)
        s.w[i] = reinterpret_cast<uint64_t*>(take(s.g.rows * 8));
    for (int i = 0; i < 2; i++)
        s.o[i] = reinterpret_cast<uint64_t*>(take(s.g.out_rows * 8));
    const size_t nt = s.g.rows / MN_TS;
    s.tiles = reinterpret_cast<RunSum*>(take(nt * sizeof(RunSum)));
    s.carry = reinterpret_cast<RunSum*>(take(nt * sizeof(RunSum)));
    s.counts = reinterpret_cast<uint32_t*>(take((s.g.rows >> OP_LT) * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take(((s.g.rows >> OP_LT) + 1) * 4));
    s.n_marked = reinterpret_cast<uint64_t*>(take(8));
    s.ocounts = reinterpret_cast<uint32_t*>(take((s.g.out_rows >> OP_LT) * 4));
    s.oprefix = reinterpret_cast<uint32_t*>(take(((s.g.out_rows >> OP_LT) + 1) * 4));
    s.pairs = reinterpret_cast<uint64_t*>(take(8));
    s.stat = reinterpret_cast<unsigned long long*>(take(16));
    s.bytes = off;
    return s;
}

using HjRec = RowRec<2, 1, false, KEY_FULL>;

} // namespace velo

extern "C" size_t velo_ohash_join_scratch_bytes(size_t build_n, size_t probe_n)
{
    return hj_layout(nullptr, build_n, probe_n).bytes;
}

extern "C" velo_status velo_ohash_join(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                                       const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n,
                                       uint32_t key_type, uint64_t hash_seed, int64_t* d_out_build_rowid,
                                       int64_t* d_out_probe_rowid, uint64_t* d_counts, void* d_scratch,
                                       size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_counts)
        return einval("velo_ohash_join: null counts");
    if (key_type != VELO_INTEGER && key_type != VELO_BIGINT)
        return einval("velo_ohash_join: join keys must be INTEGER or BIGINT");
    if (build_n >= 0x80000000ull || probe_n >= 0x80000000ull)
        return einval("velo_ohash_join: sizes must be below 2^31");
    if (probe_n == 0 || build_n == 0) {
        VELO_CUDA_TRY(cudaMemsetAsync(d_counts, 0, 24, st), "cudaMemsetAsync");
        if (probe_n) {
            VELO_CUDA_TRY(cudaMemsetAsync(d_out_build_rowid, 0xFF, probe_n * 8, st), "cudaMemsetAsync");
            VELO_CUDA_TRY(cudaMemsetAsync(d_out_probe_rowid, 0xFF, probe_n * 8, st), "cudaMemsetAsync");
        }
        return VELO_OK;
    }
    if (!d_build_keys || !d_probe_keys || !d_out_build_rowid || !d_out_probe_rowid)
        return einval("velo_ohash_join: null buffer");
    HjScratch s = hj_layout(static_cast<char*>(d_scratch), build_n, probe_n);
    const HjGeom& g = s.g;
    const int logR = ilog2_floor(g.rows), logO = ilog2_floor(g.out_rows);
    if (logR > MAX_LOGN)
        return einval("velo_ohash_join: too large");
    if ((size_t)g.cb * 16 > MAX_SMEM_BYTES)
        return einval("velo_ohash_join: bins too large");
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ohash_join: scratch must hold velo_ohash_join_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    VELO_CUDA_TRY(cudaMemsetAsync(s.stat, 0, 16, st), "cudaMemsetAsync");
    k_hj_pack<<<mn_grid(g.rows), 256, 0, st>>>(d_build_keys, d_build_mask, build_n, d_probe_keys, d_probe_mask,
                                               probe_n, key_type == VELO_BIGINT, g, hash_seed, s.w[0], s.w[1]);
    VELO_CUDA_TRY(cudaGetLastError(), "ohash_join pack launch");
    HjRec::Cols c;
    for (int i = 0; i < 2; i++) {
        c.w[i] = s.w[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = ~0ull;
    c.mark_word = 0;
    c.mark_bit = 63;
    c.mark_inv = 1; // kept rows (bit 63 clear) are marked
    std::vector<NetPass> passes;
    plan_sort(logR, OP_LT, OP_LMAX, passes);
    velo_status rc = launch_net12<HjRec>(c, NetGeom { g.rows, logR, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    const int nt = (int)(g.rows / MN_TS);
    k_hj_sum<<<nt, MN_THREADS, 0, st>>>(s.w[0], s.tiles);
    k_run_scan<<<1, 1024, 0, st>>>(s.tiles, nt, s.carry);
    k_hj_rank<<<nt, MN_THREADS, 0, st>>>(s.w[0], s.carry, g.B, g.cb, g.cp, s.stat + 1);
    VELO_CUDA_TRY(cudaGetLastError(), "ohash_join rank launch");
    const int nct = (int)(g.rows >> OP_LT);
    k_count_marks<HjRec><<<nct, 256, 0, st>>>(c, g.rows, OP_LT, s.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, nct, s.prefix, s.n_marked);
    passes.clear();
    plan_compact(logR, OP_LT, OP_LMAX, passes);
    rc = launch_net12<HjRec>(c, NetGeom { g.rows, logR, 0 }, passes, s.prefix, st);
    if (rc != VELO_OK)
        return rc;
    const size_t smem = (size_t)g.cb * 16;
    static int done[64] = {};
    rc = ensure_smem(k_hj_bins, MAX_SMEM_BYTES, done);
    if (rc != VELO_OK)
        return rc;
    k_hj_bins<<<g.B, HJ_THREADS, smem, st>>>(s.w[0], s.w[1], g, g.out_rows, s.o[0], s.o[1], s.stat);
    VELO_CUDA_TRY(cudaGetLastError(), "ohash_join bins launch");
    HjRec::Cols oc;
    for (int i = 0; i < 2; i++) {
        oc.w[i] = s.o[i];
        oc.pad[i] = ~0ull;
    }
    oc.mask[0] = ~0ull;
    oc.mark_word = 0;
    oc.mark_bit = 63;
    oc.mark_inv = 1; // joined probe slots
    const int nco = (int)(g.out_rows >> OP_LT);
    k_count_marks<HjRec><<<nco, 256, 0, st>>>(oc, g.out_rows, OP_LT, s.ocounts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.ocounts, nco, s.oprefix, s.pairs);
    passes.clear();
    plan_compact(logO, OP_LT, OP_LMAX, passes);
    rc = launch_net12<HjRec>(oc, NetGeom { g.out_rows, logO, 0 }, passes, s.oprefix, st);
    if (rc != VELO_OK)
        return rc;
    k_hj_out<<<mn_grid(probe_n), 256, 0, st>>>(s.o[0], s.o[1], probe_n, s.pairs, s.stat, s.stat + 1,
                                               d_out_build_rowid, d_out_probe_rowid, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "ohash_join out launch");
    return VELO_OK;
}
