// Column-level entry points used by the C++ operator layer:
//   velo_range_mask        conjunctive range predicate -> u8 mask (the
//                          pushed-down WHERE of SeqScanOperator evaluated on
//                          the device, src/operator/seq_scan_operator.cpp:38-45)
//   velo_iota_i64          row ids (the $_rowid column of a scan)
//   velo_ocompact_columns  oblivious in-place compaction of typed columns and
//                          their validity bytes by a mask: the ORCompact
//                          network replaces OP_SCATTER + OP_GATHER of
//                          FilterCompactionOperator::processBatchOnGpu
//                          (src/operator/filter_compaction_operator.cpp:65-184)
//
// velo_ocompact_columns packs two columns per record (values zero-extended to
// u64 words 0 and 1; word 2 = mark | validity bits) and runs the ORCompact
// passes once per pair of columns.  The network's exchanges depend only on
// the marks and the public row count, so every pair is moved by the same
// permutation: the marked rows, in input order, first.
#include "net_impl.cuh"

namespace velo {

using ColRec = RowRec<3, 1, false>;
constexpr int COL_LT = 12; // 4096-row tiles (CTA shape per record width: Tile12)

__device__ __forceinline__ uint64_t load_bits(const void* p, int bytes, size_t i)
{
    switch (bytes) {
    case 1:
        return static_cast<const uint8_t*>(p)[i];
    case 2:
        return static_cast<const uint16_t*>(p)[i];
    case 4:
        return static_cast<const uint32_t*>(p)[i];
    default:
        return static_cast<const uint64_t*>(p)[i];
    }
}

__device__ __forceinline__ void store_bits(void* p, int bytes, size_t i, uint64_t v)
{
    switch (bytes) {
    case 1:
        static_cast<uint8_t*>(p)[i] = (uint8_t)v;
        break;
    case 2:
        static_cast<uint16_t*>(p)[i] = (uint16_t)v;
        break;
    case 4:
        static_cast<uint32_t*>(p)[i] = (uint32_t)v;
        break;
    default:
        static_cast<uint64_t*>(p)[i] = v;
    }
}

// value of an integer column as int64 (DATE is an unsigned day count)
__device__ __forceinline__ int64_t load_int(const void* p, uint32_t type, size_t i)
{
    switch (type) {
    case VELO_TINYINT:
        return static_cast<const int8_t*>(p)[i];
    case VELO_SMALLINT:
        return static_cast<const int16_t*>(p)[i];
    case VELO_INTEGER:
        return static_cast<const int32_t*>(p)[i];
    case VELO_DATE:
        return static_cast<const uint32_t*>(p)[i];
    case VELO_BOOLEAN:
        return static_cast<const uint8_t*>(p)[i];
    default:
        return static_cast<const int64_t*>(p)[i];
    }
}

__global__ void k_range_mask(const void* col, uint32_t type, size_t n, int64_t lo, int64_t hi, uint8_t* mask,
                             int combine)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_range_mask"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const int64_t v = load_int(col, type, i);
        const uint8_t in = (v >= lo) & (v <= hi);
        mask[i] = combine ? (uint8_t)(mask[i] & in) : in;
    }
}

__global__ void k_iota_i64(int64_t* out, size_t n, int64_t start)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_iota_i64"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x)
        out[i] = start + (int64_t)i;
}

// per-tile counts of marked rows (rows >= n unmarked)
__global__ void __launch_bounds__(256) k_mask_tile_counts(const uint8_t* mask, size_t n, int lt, uint32_t* counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_mask_tile_counts"));
    __shared__ uint32_t tmp[33];
    const size_t base = (size_t)blockIdx.x << lt;
    uint32_t cnt = 0;
    for (int i = threadIdx.x; i < (1 << lt); i += blockDim.x) {
        const size_t g = base + i;
        cnt += (g < n && mask[g] != 0) ? 1u : 0u;
    }
    uint32_t total;
    block_exclusive_scan(cnt, tmp, &total);
    if (threadIdx.x == 0)
        counts[blockIdx.x] = total;
}

struct ColPair {
    const void* a;
    const void* b;
    const uint8_t* va;
    const uint8_t* vb;
    int ba, bb; // value bytes (0: absent)
};

__global__ void k_pack_pair(ColPair p, const uint8_t* mask, size_t n, size_t np, uint64_t* w0, uint64_t* w1,
                            uint64_t* w2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_pack_pair"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, np); i += (size_t)gridDim.x * blockDim.x) {
        uint64_t a = 0, b = 0, m = 0;
        if (i < n) {
            a = p.ba ? load_bits(p.a, p.ba, i) : 0;
            b = p.bb ? load_bits(p.b, p.bb, i) : 0;
            const uint64_t va = p.va ? (p.va[i] != 0) : 1, vb = p.vb ? (p.vb[i] != 0) : 1;
            m = (uint64_t)(mask[i] != 0) | (va << 8) | (vb << 16);
        }
        w0[i] = a;
        w1[i] = b;
        w2[i] = m;
    }
}

struct ColPairOut {
    void* a;
    void* b;
    uint8_t* va;
    uint8_t* vb;
    int ba, bb;
};

__global__ void k_unpack_pair(ColPairOut p, size_t n, const uint64_t* w0, const uint64_t* w1, const uint64_t* w2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_unpack_pair"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t m = w2[i];
        if (p.ba)
            store_bits(p.a, p.ba, i, w0[i]);
        if (p.bb)
            store_bits(p.b, p.bb, i, w1[i]);
        if (p.va)
            p.va[i] = (uint8_t)((m >> 8) & 1);
        if (p.vb)
            p.vb[i] = (uint8_t)((m >> 16) & 1);
    }
}

struct ColScratch {
    uint64_t* w[3];
    uint8_t* mask;
    uint32_t* counts;
    uint32_t* prefix;
    size_t bytes;
    size_t np;
    int ntiles;
};

static ColScratch col_layout(char* base, size_t n)
{
    ColScratch s {};
    size_t np = next_pow2(n);
    if (np < ((size_t)1 << COL_LT))
        np = (size_t)1 << COL_LT;
    s.np = np;
    s.ntiles = (int)(np >> COL_LT);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes, 256);
        return p;
    };
    for (int i = 0; i < 3; i++)
        s.w[i] = reinterpret_cast<uint64_t*>(take(np * 8));
    s.mask = reinterpret_cast<uint8_t*>(take(n ? n : 1));
    s.counts = reinterpret_cast<uint32_t*>(take((size_t)s.ntiles * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take(((size_t)s.ntiles + 1) * 4));
    s.bytes = off;
    return s;
}

static unsigned grid_for(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

} // namespace velo

using namespace velo;

extern "C" velo_status velo_range_mask(const void* d_col, uint32_t type, size_t n, int64_t lo, int64_t hi,
                                       uint8_t* d_mask, uint32_t combine, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_col || !d_mask)
        return einval("velo_range_mask: null argument");
    if (type == VELO_FLOAT || type == VELO_DOUBLE || type == VELO_VARCHAR || type_bytes(type) == 0)
        return einval("velo_range_mask: integer or DATE column expected");
    k_range_mask<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_col, type, n, lo, hi, d_mask, combine ? 1 : 0);
    VELO_CUDA_TRY(cudaGetLastError(), "range mask launch");
    return VELO_OK;
}

extern "C" velo_status velo_iota_i64(int64_t* d_out, size_t n, int64_t start, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_out)
        return einval("velo_iota_i64: null argument");
    k_iota_i64<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_out, n, start);
    VELO_CUDA_TRY(cudaGetLastError(), "iota launch");
    return VELO_OK;
}

extern "C" size_t velo_ocompact_columns_scratch_bytes(size_t n) { return col_layout(nullptr, n).bytes; }

extern "C" velo_status velo_ocompact_columns(void* const* d_cols, const uint32_t* types, uint8_t* const* d_valid,
                                             uint32_t n_cols, const uint8_t* d_mask, size_t n, uint64_t* d_count,
                                             void* d_scratch, size_t scratch_bytes, void* stream)
{
    if (!d_mask || !d_count || (n_cols && (!d_cols || !types)))
        return einval("velo_ocompact_columns: null argument");
    if (n == 0) {
        VELO_CUDA_TRY(cudaMemsetAsync(d_count, 0, 8, (cudaStream_t)stream), "cudaMemsetAsync");
        return VELO_OK;
    }
    if (next_pow2(n) > ((size_t)1 << MAX_LOGN))
        return einval("velo_ocompact_columns: n above 2^31");
    for (uint32_t c = 0; c < n_cols; c++)
        if (!d_cols[c] || type_bytes(types[c]) == 0)
            return einval("velo_ocompact_columns: null column or unknown type");
    ColScratch s = col_layout(static_cast<char*>(d_scratch), n);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ocompact_columns: scratch must hold velo_ocompact_columns_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int logN = ilog2_floor(s.np);
    // the mask may itself be one of the columns: keep the original marks
    VELO_CUDA_TRY(cudaMemcpyAsync(s.mask, d_mask, n, cudaMemcpyDeviceToDevice, st), "cudaMemcpyAsync");
    k_mask_tile_counts<<<s.ntiles, 256, 0, st>>>(s.mask, n, COL_LT, s.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, s.ntiles, s.prefix, d_count);
    VELO_CUDA_TRY(cudaGetLastError(), "mask count launch");
    std::vector<NetPass> passes;
    plan_compact(logN, COL_LT, COL_LT - 5 < 8 ? COL_LT - 5 : 8, passes);
    ColRec::Cols rc;
    for (int i = 0; i < 3; i++) {
        rc.w[i] = s.w[i];
        rc.pad[i] = 0;
    }
    rc.mask[0] = ~0ull;
    rc.mark_bit = 0;
    rc.mark_inv = 0;
    rc.mark_word = 2;
    const uint32_t groups = n_cols ? (n_cols + 1) / 2 : 0;
    for (uint32_t g = 0; g < groups; g++) {
        const uint32_t ca = 2 * g, cb = 2 * g + 1;
        ColPair in {};
        ColPairOut out {};
        in.a = out.a = d_cols[ca];
        in.ba = out.ba = type_bytes(types[ca]);
        in.va = out.va = d_valid ? d_valid[ca] : nullptr;
        if (cb < n_cols) {
            in.b = out.b = d_cols[cb];
            in.bb = out.bb = type_bytes(types[cb]);
            in.vb = out.vb = d_valid ? d_valid[cb] : nullptr;
        }
        k_pack_pair<<<grid_for(s.np), 256, 0, st>>>(in, s.mask, n, s.np, s.w[0], s.w[1], s.w[2]);
        VELO_CUDA_TRY(cudaGetLastError(), "column pack launch");
        velo_status rc2 = launch_net12<ColRec>(rc, NetGeom { s.np, logN, 0 }, passes, s.prefix, st);
        if (rc2 != VELO_OK)
            return rc2;
        k_unpack_pair<<<grid_for(n), 256, 0, st>>>(out, n, s.w[0], s.w[1], s.w[2]);
        VELO_CUDA_TRY(cudaGetLastError(), "column unpack launch");
    }
    return VELO_OK;
}

// ---------------------------------------------------------------------------
// typed oblivious gather with validity (materialization of one column)
// ---------------------------------------------------------------------------

namespace velo {

// table column -> u64 words: 4-byte and smaller values carry their validity
// in bit 32; 8-byte values are widened alone (validity gathered separately)
__global__ void k_widen_col(const void* col, int bytes, const uint8_t* valid, size_t n, uint64_t* out)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_widen_col"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t v = load_bits(col, bytes, i);
        const uint64_t ok = valid ? (valid[i] != 0) : 1;
        out[i] = bytes < 8 ? (v | (ok << 32)) : v;
    }
}

__global__ void k_widen_valid(const uint8_t* valid, size_t n, uint64_t* out)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_widen_valid"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x)
        out[i] = valid ? (valid[i] != 0) : 1;
}

// row ids -> u32 request ids; negative or >= table_n requests no row
__global__ void k_rowids_u32(const int64_t* rid, size_t n, size_t table_n, uint32_t* out)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_rowids_u32"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const int64_t r = rid[i];
        out[i] = (r >= 0 && (uint64_t)r < table_n) ? (uint32_t)r : 0xFFFFFFFFu;
    }
}

__global__ void k_narrow_col(const uint64_t* w, size_t n, int bytes, void* out, uint8_t* out_valid)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_narrow_col"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t x = w[i];
        store_bits(out, bytes, i, bytes < 8 ? (x & 0xFFFFFFFFull) : x);
        if (bytes < 8 && out_valid)
            out_valid[i] = (uint8_t)((x >> 32) & 1);
    }
}

__global__ void k_narrow_valid(const uint64_t* w, size_t n, uint8_t* out_valid)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_narrow_valid"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x)
        out_valid[i] = (uint8_t)(w[i] & 1);
}

struct GatherColScratch {
    uint64_t* table;
    uint32_t* rids;
    uint64_t* out;
    char* inner;
    size_t inner_bytes;
    size_t bytes;
};

static GatherColScratch gather_col_layout(char* base, size_t table_n, size_t n)
{
    GatherColScratch s {};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes ? bytes : 1, 256);
        return p;
    };
    s.table = reinterpret_cast<uint64_t*>(take(table_n * 8));
    s.rids = reinterpret_cast<uint32_t*>(take(n * 4));
    s.out = reinterpret_cast<uint64_t*>(take(n * 8));
    s.inner_bytes = velo_ogather_scratch_bytes(table_n, n);
    s.inner = take(s.inner_bytes);
    s.bytes = off;
    return s;
}

} // namespace velo

extern "C" size_t velo_ogather_column_scratch_bytes(size_t table_n, size_t n)
{
    return gather_col_layout(nullptr, table_n, n).bytes;
}

extern "C" velo_status velo_ogather_column(const void* d_table_col, uint32_t type, const uint8_t* d_table_valid,
                                           size_t table_n, const int64_t* d_rowids, size_t n, void* d_out,
                                           uint8_t* d_out_valid, void* d_scratch, size_t scratch_bytes, void* stream)
{
    if (n == 0)
        return VELO_OK;
    const int bytes = type_bytes(type);
    if (!d_table_col || !d_rowids || !d_out || bytes == 0)
        return einval("velo_ogather_column: null argument or unknown type");
    if (table_n >= 0xFFFFFFFFull || n >= 0xFFFFFFFFull)
        return einval("velo_ogather_column: sizes must fit 32 bits");
    GatherColScratch s = gather_col_layout(static_cast<char*>(d_scratch), table_n, n);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ogather_column: scratch must hold velo_ogather_column_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    k_rowids_u32<<<grid_for(n), 256, 0, st>>>(d_rowids, n, table_n, s.rids);
    if (table_n)
        k_widen_col<<<grid_for(table_n), 256, 0, st>>>(d_table_col, bytes, d_table_valid, table_n, s.table);
    VELO_CUDA_TRY(cudaGetLastError(), "gather column pack launch");
    velo_status rc = velo_ogather_u64(s.table, table_n, s.rids, n, s.out, s.inner, s.inner_bytes, stream);
    if (rc != VELO_OK)
        return rc;
    k_narrow_col<<<grid_for(n), 256, 0, st>>>(s.out, n, bytes, d_out, d_out_valid);
    VELO_CUDA_TRY(cudaGetLastError(), "gather column unpack launch");
    if (bytes == 8 && d_out_valid) {
        if (table_n)
            k_widen_valid<<<grid_for(table_n), 256, 0, st>>>(d_table_valid, table_n, s.table);
        rc = velo_ogather_u64(s.table, table_n, s.rids, n, s.out, s.inner, s.inner_bytes, stream);
        if (rc != VELO_OK)
            return rc;
        k_narrow_valid<<<grid_for(n), 256, 0, st>>>(s.out, n, d_out_valid);
        VELO_CUDA_TRY(cudaGetLastError(), "gather validity launch");
    }
    return VELO_OK;
}

// ---------------------------------------------------------------------------
// integer column -> int64 (operands of SUM)
// ---------------------------------------------------------------------------

namespace velo {
__global__ void k_widen_i64(const void* col, uint32_t type, size_t n, int64_t* out)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_widen_i64"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n);
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = load_int(col, type, i);
}
} // namespace velo

extern "C" velo_status velo_widen_i64(const void* d_col, uint32_t type, size_t n, int64_t* d_out, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_col || !d_out)
        return einval("velo_widen_i64: null argument");
    if (type == VELO_FLOAT || type == VELO_DOUBLE || type == VELO_VARCHAR || type_bytes(type) == 0)
        return einval("velo_widen_i64: integer, BOOLEAN or DATE column expected");
    k_widen_i64<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_col, type, n, d_out);
    VELO_CUDA_TRY(cudaGetLastError(), "widen launch");
    return VELO_OK;
}
