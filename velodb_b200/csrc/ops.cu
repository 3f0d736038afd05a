// Column operators of the reference's command set and their oblivious
// replacements:
//   compat (reference semantics, data-dependent addresses as in the
//   reference):  OP_PERMUTE, OP_SCATTER, OP_GATHER, OP_COMPARE_EQ,
//                OP_COMPOSE_POSITION_MAP, OP_ENRICH_POSITIONS
//   oblivious:   position-map shuffle (device PRF + bitonic network),
//                oblivious gather (union sort + fill + sort back),
//                PK-FK equi-join producing (build rowid, probe rowid) pairs
#include "ops.cuh"

namespace velo {

static unsigned grid_for(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

// ---------------------------------------------------------------------------
// kernels of the plain path: each runs the body of ops.cuh / union.cuh over
// its grid
// ---------------------------------------------------------------------------

template <typename T>
__global__ void k_permute(T* out, const T* in, const int64_t* idx, size_t n)
{
    permute_body(out, in, idx, n, blockIdx.x, gridDim.x);
}

template <typename T>
__global__ void k_gather(T* out, const T* in, const int32_t* idx, const uint8_t* mask, size_t n)
{
    gather_body(out, in, idx, mask, n, blockIdx.x, gridDim.x);
}

template <typename T>
__global__ void k_compare_eq(const T* l, const T* r, uint8_t* out, size_t n)
{
    compare_eq_body(l, r, out, n, blockIdx.x, gridDim.x);
}

__global__ void k_fill_u8(uint8_t* out, uint8_t v, size_t n)
{
    fill_u8_body(out, v, n, blockIdx.x, gridDim.x);
}

__global__ void k_compose(const uint32_t* old_map, const uint32_t* sigma, uint32_t* new_map, size_t n)
{
    compose_body(old_map, sigma, new_map, n, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256) k_scatter_count(const uint8_t* mask, size_t n, uint32_t* counts)
{
    __shared__ uint32_t tmp[33];
    scatter_count_tile(mask, n, counts, blockIdx.x, tmp);
}

__global__ void __launch_bounds__(256) k_scatter_write(const uint8_t* mask, size_t n, const uint32_t* prefix,
                                                       int32_t* out_idx)
{
    __shared__ uint32_t tmp[33];
    scatter_write_tile(mask, n, prefix, out_idx, blockIdx.x, tmp);
}

__global__ void k_shuffle_pack(const uint32_t* map, size_t n, size_t np, uint64_t counter, uint64_t key, uint64_t* k,
                               uint32_t* p)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_shuffle_pack"));
    shuffle_pack_body(map, n, np, counter, key, k, p, blockIdx.x, gridDim.x);
}

__global__ void k_copy_u32(uint32_t* dst, const uint32_t* src, size_t n)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_copy_u32"));
    copy_u32_body(dst, src, n, blockIdx.x, gridDim.x);
}

// exclusive scan of the tile carries; one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_fill_scan(const FillCarry* tile_last, int ntiles, FillCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_scan"));
    __shared__ FillCarry wsm[33];
    fill_scan_body(tile_last, ntiles, carry, wsm);
}

__global__ void k_ogather_pack(const uint64_t* table, size_t tn, const uint32_t* rids, size_t rn, size_t rows,
                               uint64_t* w0, uint64_t* w1, uint64_t* w2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_ogather_pack"));
    ogather_pack_body(table, tn, rids, rn, rows, w0, w1, w2, blockIdx.x, gridDim.x);
}

__global__ void k_ogather_out(const uint64_t* w1, size_t rn, uint64_t* out)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_ogather_out"));
    ogather_out_body(w1, rn, out, blockIdx.x, gridDim.x);
}

__global__ void k_ojoin_pack(const void* bk, const uint8_t* bm, size_t bn, const void* pk, const uint8_t* pm, size_t pn,
                             int key64, size_t rows, uint64_t* w0, uint64_t* w1, uint64_t* w2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_ojoin_pack"));
    ojoin_pack_body(bk, bm, bn, pk, pm, pn, key64, rows, w0, w1, w2, blockIdx.x, gridDim.x);
}

__global__ void k_ojoin_out(const uint64_t* w1, const uint64_t* w2, size_t pn, int64_t* ob, int64_t* op)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_ojoin_out"));
    ojoin_out_body(w1, w2, pn, ob, op, blockIdx.x, gridDim.x);
}

__global__ void k_zero_u64(unsigned long long* p, int n)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_zero_u64"));
    if ((int)threadIdx.x < n)
        p[threadIdx.x] = 0;
}

__global__ void k_join_counts(const uint64_t* n_joined, const unsigned long long* dups, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_join_counts"));
    join_counts_body(n_joined, dups, d_counts);
}

} // namespace velo

using namespace velo;

// ---- compat entry points ---------------------------------------------------

extern "C" velo_status velo_permute(void* d_out, const void* d_in, const int64_t* d_indices, size_t n, uint32_t type,
                                    void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0)
        return VELO_OK;
    if (!d_out || !d_in || !d_indices)
        return einval("velo_permute: null buffer");
    switch (type_bytes(type)) {
    case 1:
        k_permute<uint8_t><<<grid_for(n), 256, 0, st>>>((uint8_t*)d_out, (const uint8_t*)d_in, d_indices, n);
        break;
    case 2:
        k_permute<uint16_t><<<grid_for(n), 256, 0, st>>>((uint16_t*)d_out, (const uint16_t*)d_in, d_indices, n);
        break;
    case 4:
        k_permute<uint32_t><<<grid_for(n), 256, 0, st>>>((uint32_t*)d_out, (const uint32_t*)d_in, d_indices, n);
        break;
    case 8:
        k_permute<uint64_t><<<grid_for(n), 256, 0, st>>>((uint64_t*)d_out, (const uint64_t*)d_in, d_indices, n);
        break;
    default:
        return einval("velo_permute: unsupported type");
    }
    VELO_CUDA_TRY(cudaGetLastError(), "permute launch");
    return VELO_OK;
}

extern "C" velo_status velo_gather(void* d_out, const void* d_in, const int32_t* d_indices, const uint8_t* d_mask,
                                   size_t n, uint32_t type, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0)
        return VELO_OK;
    if (!d_out || !d_in || !d_indices)
        return einval("velo_gather: null buffer");
    switch (type_bytes(type)) {
    case 1:
        k_gather<uint8_t><<<grid_for(n), 256, 0, st>>>((uint8_t*)d_out, (const uint8_t*)d_in, d_indices, d_mask, n);
        break;
    case 2:
        k_gather<uint16_t><<<grid_for(n), 256, 0, st>>>((uint16_t*)d_out, (const uint16_t*)d_in, d_indices, d_mask, n);
        break;
    case 4:
        k_gather<uint32_t><<<grid_for(n), 256, 0, st>>>((uint32_t*)d_out, (const uint32_t*)d_in, d_indices, d_mask, n);
        break;
    case 8:
        k_gather<uint64_t><<<grid_for(n), 256, 0, st>>>((uint64_t*)d_out, (const uint64_t*)d_in, d_indices, d_mask, n);
        break;
    default:
        return einval("velo_gather: unsupported type");
    }
    VELO_CUDA_TRY(cudaGetLastError(), "gather launch");
    return VELO_OK;
}

extern "C" size_t velo_scatter_scratch_bytes(size_t n)
{
    const size_t nt = (n + (1 << SC_LT) - 1) >> SC_LT;
    return align_up((nt ? nt : 1) * 4, 256) + align_up(((nt ? nt : 1) + 1) * 4, 256);
}

extern "C" velo_status velo_scatter(const uint8_t* d_mask, size_t n, int32_t* d_out_indices, uint64_t* d_count,
                                    void* d_scratch, size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_count)
        return einval("velo_scatter: null count");
    if (n == 0) {
        VELO_CUDA_TRY(cudaMemsetAsync(d_count, 0, 8, st), "cudaMemsetAsync");
        return VELO_OK;
    }
    if (!d_mask || !d_out_indices)
        return einval("velo_scatter: null buffer");
    if (!d_scratch || scratch_bytes < velo_scatter_scratch_bytes(n)) {
        set_error("velo_scatter: scratch must hold velo_scatter_scratch_bytes(n) bytes");
        return VELO_ENOMEM;
    }
    const size_t nt = (n + (1 << SC_LT) - 1) >> SC_LT;
    uint32_t* counts = static_cast<uint32_t*>(d_scratch);
    uint32_t* prefix = reinterpret_cast<uint32_t*>(static_cast<char*>(d_scratch) + align_up(nt * 4, 256));
    k_scatter_count<<<(unsigned)nt, 256, 0, st>>>(d_mask, n, counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(counts, (int)nt, prefix, d_count);
    k_scatter_write<<<(unsigned)nt, 256, 0, st>>>(d_mask, n, prefix, d_out_indices);
    VELO_CUDA_TRY(cudaGetLastError(), "scatter launch");
    return VELO_OK;
}

extern "C" velo_status velo_compare_eq(const void* d_left, const void* d_right, uint8_t* d_out_mask, size_t n,
                                       uint32_t type, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0)
        return VELO_OK;
    if (!d_left || !d_right || !d_out_mask)
        return einval("velo_compare_eq: null buffer");
    const unsigned g = grid_for(n);
    switch (type) {
    case VELO_TINYINT:
        k_compare_eq<int8_t><<<g, 256, 0, st>>>((const int8_t*)d_left, (const int8_t*)d_right, d_out_mask, n);
        break;
    case VELO_SMALLINT:
        k_compare_eq<int16_t><<<g, 256, 0, st>>>((const int16_t*)d_left, (const int16_t*)d_right, d_out_mask, n);
        break;
    case VELO_INTEGER:
    case VELO_DATE:
        k_compare_eq<int32_t><<<g, 256, 0, st>>>((const int32_t*)d_left, (const int32_t*)d_right, d_out_mask, n);
        break;
    case VELO_BIGINT:
        k_compare_eq<int64_t><<<g, 256, 0, st>>>((const int64_t*)d_left, (const int64_t*)d_right, d_out_mask, n);
        break;
    case VELO_FLOAT:
        k_compare_eq<float><<<g, 256, 0, st>>>((const float*)d_left, (const float*)d_right, d_out_mask, n);
        break;
    case VELO_DOUBLE:
        k_compare_eq<double><<<g, 256, 0, st>>>((const double*)d_left, (const double*)d_right, d_out_mask, n);
        break;
    default:
        // unsupported types compare as all-false, as the reference does
        k_fill_u8<<<g, 256, 0, st>>>(d_out_mask, 0, n);
        break;
    }
    VELO_CUDA_TRY(cudaGetLastError(), "compare launch");
    return VELO_OK;
}

extern "C" velo_status velo_compose_position_map(const uint32_t* d_old, const uint32_t* d_sigma, uint32_t* d_new,
                                                 size_t n, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_old || !d_sigma || !d_new)
        return einval("velo_compose_position_map: null buffer");
    k_compose<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_old, d_sigma, d_new, n);
    VELO_CUDA_TRY(cudaGetLastError(), "compose launch");
    return VELO_OK;
}

extern "C" velo_status velo_enrich_positions(const uint32_t* d_record_ids, const uint32_t* d_map, uint32_t* d_out,
                                             size_t n, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_record_ids || !d_map || !d_out)
        return einval("velo_enrich_positions: null buffer");
    // pos[i] = map[rid[i]]: the same gather as a composition
    k_compose<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_map, d_record_ids, d_out, n);
    VELO_CUDA_TRY(cudaGetLastError(), "enrich launch");
    return VELO_OK;
}

// ---- oblivious shuffle ---------------------------------------------------------

extern "C" size_t velo_oshuffle_scratch_bytes(size_t n)
{
    const size_t np = next_pow2(n);
    return align_up(np * 8, 256) + align_up(np * 4, 256);
}

extern "C" velo_status velo_oshuffle_position_map(uint32_t* d_map, size_t n, uint64_t key, uint64_t counter,
                                                  void* d_scratch, size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0)
        return VELO_OK;
    if (!d_map)
        return einval("velo_oshuffle_position_map: null map");
    const size_t np = next_pow2(n);
    if (np > ((size_t)1 << MAX_LOGN))
        return einval("velo_oshuffle_position_map: n too large");
    if (!d_scratch || scratch_bytes < velo_oshuffle_scratch_bytes(n)) {
        set_error("velo_oshuffle_position_map: scratch must hold velo_oshuffle_scratch_bytes(n) bytes");
        return VELO_ENOMEM;
    }
    uint64_t* k = static_cast<uint64_t*>(d_scratch);
    uint32_t* p = reinterpret_cast<uint32_t*>(static_cast<char*>(d_scratch) + align_up(np * 8, 256));
    k_shuffle_pack<<<grid_for(np), 256, 0, st>>>(d_map, n, np, counter, key, k, p);
    VELO_CUDA_TRY(cudaGetLastError(), "shuffle pack launch");
    velo_status rc = velo_osort_kp(k, p, np, np, nullptr, stream);
    if (rc != VELO_OK)
        return rc;
    k_copy_u32<<<grid_for(n), 256, 0, st>>>(d_map, p, n);
    VELO_CUDA_TRY(cudaGetLastError(), "shuffle copy launch");
    return VELO_OK;
}

// ---- oblivious gather ----------------------------------------------------------

extern "C" size_t velo_ogather_scratch_bytes(size_t table_n, size_t n_req)
{
    return union_layout(nullptr, union_rows(table_n + n_req)).bytes;
}

extern "C" velo_status velo_ogather_u64(const uint64_t* d_table, size_t table_n, const uint32_t* d_rids, size_t n_req,
                                        uint64_t* d_out, void* d_scratch, size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n_req == 0)
        return VELO_OK;
    if (!d_table || !d_rids || !d_out)
        return einval("velo_ogather_u64: null buffer");
    if (table_n >= 0xFFFFFFFFull || n_req >= 0xFFFFFFFFull)
        return einval("velo_ogather_u64: sizes must fit 32 bits");
    const size_t rows = union_rows(table_n + n_req);
    const int logR = ilog2_floor(rows);
    if (logR > MAX_LOGN)
        return einval("velo_ogather_u64: too large");
    UnionScratch s = union_layout(static_cast<char*>(d_scratch), rows);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ogather_u64: scratch must hold velo_ogather_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    k_ogather_pack<<<grid_for(rows), 256, 0, st>>>(d_table, table_n, d_rids, n_req, rows, s.w[0], s.w[1], s.w[2]);
    VELO_CUDA_TRY(cudaGetLastError(), "ogather pack launch");
    Rec3::Cols c;
    for (int i = 0; i < 3; i++) {
        c.w[i] = s.w[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = 0xFFFFFFFF80000000ull;
    c.mark_bit = 0;
    c.mark_inv = 0;
    c.mark_word = 0;
    std::vector<NetPass> passes;
    plan_sort(logR, OP_LT, OP_LMAX, passes);
    velo_status rc = launch_net12<Rec3>(c, NetGeom { rows, logR, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    rc = run_fill<GatherFill>(s.w[0], s.w[1], s.w[2], rows, s.tl, s.carry, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    c.mask[0] = ~0ull;
    rc = launch_net12<Rec3>(c, NetGeom { rows, logR, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    k_ogather_out<<<grid_for(n_req), 256, 0, st>>>(s.w[1], n_req, d_out);
    VELO_CUDA_TRY(cudaGetLastError(), "ogather out launch");
    return VELO_OK;
}

// ---- oblivious PK-FK join ------------------------------------------------------

extern "C" size_t velo_ojoin_scratch_bytes(size_t build_n, size_t probe_n)
{
    return union_layout(nullptr, union_rows(build_n + probe_n)).bytes;
}

extern "C" velo_status velo_ojoin_pkfk(const void* d_build_keys, const uint8_t* d_build_mask, size_t build_n,
                                       const void* d_probe_keys, const uint8_t* d_probe_mask, size_t probe_n,
                                       uint32_t key_type, int64_t* d_out_build_rowid, int64_t* d_out_probe_rowid,
                                       uint64_t* d_counts, void* d_scratch, size_t scratch_bytes, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_counts)
        return einval("velo_ojoin_pkfk: null counts");
    if (key_type != VELO_INTEGER && key_type != VELO_BIGINT)
        return einval("velo_ojoin_pkfk: join keys must be INTEGER or BIGINT");
    if (probe_n == 0 || build_n == 0) {
        VELO_CUDA_TRY(cudaMemsetAsync(d_counts, 0, 16, st), "cudaMemsetAsync");
        if (probe_n) {
            VELO_CUDA_TRY(cudaMemsetAsync(d_out_build_rowid, 0xFF, probe_n * 8, st), "cudaMemsetAsync");
            VELO_CUDA_TRY(cudaMemsetAsync(d_out_probe_rowid, 0xFF, probe_n * 8, st), "cudaMemsetAsync");
        }
        return VELO_OK;
    }
    if (!d_build_keys || !d_probe_keys || !d_out_build_rowid || !d_out_probe_rowid)
        return einval("velo_ojoin_pkfk: null buffer");
    const size_t rows = union_rows(build_n + probe_n);
    const int logR = ilog2_floor(rows);
    if (logR > MAX_LOGN)
        return einval("velo_ojoin_pkfk: too large");
    UnionScratch s = union_layout(static_cast<char*>(d_scratch), rows);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_ojoin_pkfk: scratch must hold velo_ojoin_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    k_zero_u64<<<1, 32, 0, st>>>(s.stat, 1);
    k_ojoin_pack<<<grid_for(rows), 256, 0, st>>>(d_build_keys, d_build_mask, build_n, d_probe_keys, d_probe_mask,
                                                 probe_n, key_type == VELO_BIGINT, rows, s.w[0], s.w[1], s.w[2]);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin pack launch");
    Rec3K2::Cols c;
    for (int i = 0; i < 3; i++) {
        c.w[i] = s.w[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = ~0ull;
    c.mask[1] = OJ_TAG;
    c.mark_word = 1;
    c.mark_bit = 61;
    c.mark_inv = 0;
    std::vector<NetPass> passes;
    plan_sort(logR, OP_LT, OP_LMAX, passes);
    velo_status rc = launch_net12<Rec3K2>(c, NetGeom { rows, logR, 0 }, passes, nullptr, st);
    if (rc != VELO_OK)
        return rc;
    rc = run_fill<JoinFill>(s.w[0], s.w[1], s.w[2], rows, s.tl, s.carry, s.stat, st);
    if (rc != VELO_OK)
        return rc;
    const int nct = (int)(rows >> OP_LT);
    k_count_marks<Rec3K2><<<nct, 256, 0, st>>>(c, rows, OP_LT, s.counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, nct, s.prefix, s.n_marked);
    std::vector<NetPass> cp;
    plan_compact(logR, OP_LT, OP_LMAX, cp);
    rc = launch_net12<Rec3K2>(c, NetGeom { rows, logR, 0 }, cp, s.prefix, st);
    if (rc != VELO_OK)
        return rc;
    k_ojoin_out<<<grid_for(probe_n), 256, 0, st>>>(s.w[1], s.w[2], probe_n, d_out_build_rowid, d_out_probe_rowid);
    k_join_counts<<<1, 1, 0, st>>>(s.n_marked, s.stat, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "ojoin out launch");
    return VELO_OK;
}
