// velo_sort_columns: the reference OP_SORT contract (multi-column, per-column
// direction, in-place sorted columns + int64 permutation) on the oblivious
// bitonic network.
//
// Each row's sort columns are encoded into an order-preserving unsigned key
// of KW 64-bit words (first column most significant; signed values flip the
// sign bit, IEEE values flip all bits when negative else the sign bit,
// descending columns are complemented), the original row index rides along
// as one more word, the records are sorted by the same network as the
// reference (so equal keys keep the reference's arrangement), and the columns
// are decoded back in place.  All three steps are streaming or network passes
// with data-independent addresses.
#include "net_impl.cuh"

namespace velo {

constexpr int MAX_SORT_COLS = 8; // MAX_SORT_COLUMNS, include/common/constants.hpp.in:17

struct ColSpec {
    void* col[MAX_SORT_COLS];
    uint32_t type[MAX_SORT_COLS];
    uint32_t asc[MAX_SORT_COLS];
    int n_cols;
};

__host__ __device__ inline int type_bits(uint32_t t)
{
    switch (t) {
    case VELO_BOOLEAN:
    case VELO_TINYINT:
        return 8;
    case VELO_SMALLINT:
        return 16;
    case VELO_INTEGER:
    case VELO_FLOAT:
    case VELO_DATE:
        return 32;
    case VELO_BIGINT:
    case VELO_DOUBLE:
    case VELO_VARCHAR:
        return 64;
    default:
        return 0;
    }
}

// raw bits of the value of column c at row g, or of its pad value
// (max() ascending / lowest() descending, include/cuda/sort.cuh:79-100)
__device__ __forceinline__ uint64_t raw_value(const ColSpec& s, int c, size_t g, bool pad)
{
    const bool asc = s.asc[c] != 0;
    switch (s.type[c]) {
    case VELO_BOOLEAN:
        return pad ? (asc ? 0xFFull : 0ull) : static_cast<const uint8_t*>(s.col[c])[g];
    case VELO_TINYINT:
        return pad ? (asc ? 0x7Full : 0x80ull) : static_cast<const uint8_t*>(s.col[c])[g];
    case VELO_SMALLINT:
        return pad ? (asc ? 0x7FFFull : 0x8000ull) : static_cast<const uint16_t*>(s.col[c])[g];
    case VELO_INTEGER:
        return pad ? (asc ? 0x7FFFFFFFull : 0x80000000ull) : static_cast<const uint32_t*>(s.col[c])[g];
    case VELO_DATE:
        return pad ? (asc ? 0xFFFFFFFFull : 0ull) : static_cast<const uint32_t*>(s.col[c])[g];
    case VELO_FLOAT:
        // FLT_MAX / -FLT_MAX
        return pad ? (asc ? 0x7F7FFFFFull : 0xFF7FFFFFull) : static_cast<const uint32_t*>(s.col[c])[g];
    case VELO_BIGINT:
        return pad ? (asc ? 0x7FFFFFFFFFFFFFFFull : 0x8000000000000000ull) : static_cast<const uint64_t*>(s.col[c])[g];
    case VELO_DOUBLE:
        // DBL_MAX / -DBL_MAX
        return pad ? (asc ? 0x7FEFFFFFFFFFFFFFull : 0xFFEFFFFFFFFFFFFFull) : static_cast<const uint64_t*>(s.col[c])[g];
    case VELO_VARCHAR:
        return pad ? (asc ? ~0ull : 0ull) : static_cast<const uint64_t*>(s.col[c])[g];
    default:
        return 0;
    }
}

__device__ __forceinline__ uint64_t encode(uint32_t t, bool asc, uint64_t raw)
{
    const int w = type_bits(t);
    const uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1);
    const uint64_t sign = 1ull << (w - 1);
    uint64_t u = raw & mask;
    switch (t) {
    case VELO_TINYINT:
    case VELO_SMALLINT:
    case VELO_INTEGER:
    case VELO_BIGINT:
        u ^= sign;
        break;
    case VELO_FLOAT:
    case VELO_DOUBLE:
        u = (u & sign) ? (~u & mask) : (u | sign);
        break;
    default:
        break;
    }
    return asc ? u : (~u & mask);
}

__device__ __forceinline__ uint64_t decode(uint32_t t, bool asc, uint64_t u)
{
    const int w = type_bits(t);
    const uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1);
    const uint64_t sign = 1ull << (w - 1);
    u = asc ? u : (~u & mask);
    switch (t) {
    case VELO_TINYINT:
    case VELO_SMALLINT:
    case VELO_INTEGER:
    case VELO_BIGINT:
        u ^= sign;
        break;
    case VELO_FLOAT:
    case VELO_DOUBLE:
        u = (u & sign) ? (u & ~sign) : (~u & mask);
        break;
    default:
        break;
    }
    return u;
}

__device__ __forceinline__ void store_raw(const ColSpec& s, int c, size_t g, uint64_t v)
{
    switch (type_bits(s.type[c])) {
    case 8:
        static_cast<uint8_t*>(s.col[c])[g] = (uint8_t)v;
        break;
    case 16:
        static_cast<uint16_t*>(s.col[c])[g] = (uint16_t)v;
        break;
    case 32:
        static_cast<uint32_t*>(s.col[c])[g] = (uint32_t)v;
        break;
    default:
        static_cast<uint64_t*>(s.col[c])[g] = v;
        break;
    }
}

// key bits are laid out MSB-first across KW words
template <int KW>
__global__ void k_pack_cols(ColSpec s, size_t n, size_t np, uint64_t* words)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_pack_cols"));
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, np); g += (size_t)gridDim.x * blockDim.x) {
        uint64_t w[KW];
#pragma unroll
        for (int i = 0; i < KW; i++)
            w[i] = 0;
        int pos = 0; // bit position from the top of word 0
        for (int c = 0; c < s.n_cols; c++) {
            const int bits = type_bits(s.type[c]);
            const uint64_t u = encode(s.type[c], s.asc[c] != 0, raw_value(s, c, g, g >= n));
            const int wi = pos >> 6, off = pos & 63; // field starts at bit (63 - off) of word wi
            const int room = 64 - off;
#pragma unroll
            for (int i = 0; i < KW; i++) {
                if (i == wi) {
                    w[i] |= bits >= room ? (u >> (bits - room)) : (u << (room - bits));
                } else if (i == wi + 1 && bits > room) {
                    w[i] |= u << (64 - (bits - room));
                }
            }
            pos += bits;
        }
#pragma unroll
        for (int i = 0; i < KW; i++)
            words[(size_t)i * np + g] = w[i];
        words[(size_t)KW * np + g] = g; // row index rides along
    }
}

template <int KW>
__global__ void k_unpack_cols(ColSpec s, size_t np, const uint64_t* words, int64_t* indices)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_unpack_cols"));
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(g, np); g += (size_t)gridDim.x * blockDim.x) {
        uint64_t w[KW];
#pragma unroll
        for (int i = 0; i < KW; i++)
            w[i] = words[(size_t)i * np + g];
        int pos = 0;
        for (int c = 0; c < s.n_cols; c++) {
            const int bits = type_bits(s.type[c]);
            const uint64_t mask = bits == 64 ? ~0ull : ((1ull << bits) - 1);
            const int wi = pos >> 6, off = pos & 63, room = 64 - off;
            uint64_t u = 0;
#pragma unroll
            for (int i = 0; i < KW; i++) {
                if (i == wi)
                    u |= bits >= room ? (w[i] << (bits - room)) : (w[i] >> (room - bits));
                else if (i == wi + 1 && bits > room)
                    u |= w[i] >> (64 - (bits - room));
            }
            store_raw(s, c, g, decode(s.type[c], s.asc[c] != 0, u & mask));
            pos += bits;
        }
        indices[g] = (int64_t)words[(size_t)KW * np + g];
    }
}

template <int KW, int LOG_NT, int LOG_E>
static velo_status sort_cols_kw(const ColSpec& s, size_t n, int logN, uint64_t* words, int64_t* indices,
                                cudaStream_t st)
{
    using R = RowRec<KW + 1, KW>;
    const size_t np = (size_t)1 << logN;
    const int threads = 256;
    const unsigned blocks = (unsigned)((np + threads - 1) / threads < 148 * 16 ? (np + threads - 1) / threads : 148 * 16);
    k_pack_cols<KW><<<blocks, threads, 0, st>>>(s, n, np, words);
    VELO_CUDA_TRY(cudaGetLastError(), "pack launch");
    typename R::Cols c;
    for (int i = 0; i <= KW; i++)
        c.w[i] = words + (size_t)i * np;
    for (int i = 0; i < KW; i++)
        c.mask[i] = ~0ull;
    for (int i = 0; i <= KW; i++)
        c.pad[i] = ~0ull; // unused: every row (real or pad) is packed explicitly
    c.mark_bit = 0;
    c.mark_inv = 0;
    c.mark_word = 0;
    if (np > 1) {
        std::vector<NetPass> passes;
        const int lt = LOG_NT + LOG_E;
        plan_sort(logN, lt, lt - 5 < 8 ? lt - 5 : 8, passes);
        // every row is materialised by the pack kernel, so n = np here
        NetGeom g { np, logN, 0 };
        velo_status rc = launch_net<R, LOG_NT, LOG_E>(c, g, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
    }
    k_unpack_cols<KW><<<blocks, threads, 0, st>>>(s, np, words, indices);
    VELO_CUDA_TRY(cudaGetLastError(), "unpack launch");
    return VELO_OK;
}

static int key_words(const uint32_t* types, uint32_t n_cols)
{
    int bits = 0;
    for (uint32_t c = 0; c < n_cols; c++) {
        const int b = type_bits(types[c]);
        if (b == 0)
            return -1;
        bits += b;
    }
    const int kw = (bits + 63) / 64;
    return kw <= 4 ? kw : 8;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_sort_scratch_bytes(const uint32_t* types, uint32_t n_cols, size_t n)
{
    if (!types || n_cols == 0 || n_cols > MAX_SORT_COLS)
        return 0;
    const int kw = key_words(types, n_cols);
    if (kw < 0)
        return 0;
    return (size_t)(kw + 1) * next_pow2(n) * sizeof(uint64_t);
}

extern "C" velo_status velo_sort_columns(void* const* d_cols, const uint32_t* types, const uint8_t* ascending,
                                         uint32_t n_cols, size_t n, size_t capacity, int64_t* d_indices,
                                         void* d_scratch, size_t scratch_bytes, void* stream)
{
    if (n_cols == 0 || n_cols > MAX_SORT_COLS || !d_cols || !types || !ascending)
        return einval("velo_sort_columns: 1..8 sort columns required");
    const int kw = key_words(types, n_cols);
    if (kw < 0)
        return einval("velo_sort_columns: unsupported column type");
    if (n == 0)
        return VELO_OK;
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_sort_columns: n too large");
    if (capacity < np)
        return einval("velo_sort_columns: capacity must be >= next_pow2(n)");
    if (!d_indices)
        return einval("velo_sort_columns: null indices");
    const size_t need = (size_t)(kw + 1) * np * sizeof(uint64_t);
    if (!d_scratch || scratch_bytes < need) {
        set_error("velo_sort_columns: scratch must hold velo_sort_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    ColSpec s {};
    s.n_cols = (int)n_cols;
    for (uint32_t c = 0; c < n_cols; c++) {
        if (!d_cols[c])
            return einval("velo_sort_columns: null column");
        s.col[c] = d_cols[c];
        s.type[c] = types[c];
        s.asc[c] = ascending[c] ? 1u : 0u;
    }
    uint64_t* words = static_cast<uint64_t*>(d_scratch);
    cudaStream_t st = (cudaStream_t)stream;
    switch (kw) {
    case 1:
        return sort_cols_kw<1, 9, 4>(s, n, logN, words, d_indices, st);
    case 2:
        return sort_cols_kw<2, 9, 4>(s, n, logN, words, d_indices, st);
    // wider records take fewer rows a thread, so the row words stay in
    // registers (W x E words under the 128-register cap)
    case 3:
        return sort_cols_kw<3, 9, 3>(s, n, logN, words, d_indices, st);
    case 4:
        return sort_cols_kw<4, 9, 2>(s, n, logN, words, d_indices, st);
    default:
        return sort_cols_kw<8, 9, 2>(s, n, logN, words, d_indices, st);
    }
}
