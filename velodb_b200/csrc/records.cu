// velo_osort_records: bitonic sort of 1..3-word records keyed on word 0.
#include "net_host.cuh"

namespace velo {

// the tile configurations compiled for record sorts (see net_inst_rec*.cu);
// a fused global pass keeps 16 contiguous rows (a 128-byte line of each word
// array), so up to LT - 4 levels
#define VELO_FOR_REC_TUNES(X)                                                                                          \
    X(8, 3)                                                                                                            \
    X(9, 3)                                                                                                            \
    X(8, 4)                                                                                                            \
    X(9, 2)

template <int W, bool STRICT>
static velo_status rec_sort(uint64_t* const* words, uint64_t mask, size_t n, int logN, int log_nt, int log_e,
                            cudaStream_t st)
{
    using R = RowRec<W, 1, STRICT>;
    typename R::Cols c;
    for (int i = 0; i < W; i++) {
        c.w[i] = words[i];
        c.pad[i] = ~0ull;
    }
    c.mask[0] = mask;
    c.mark_bit = 0;
    c.mark_inv = 0;
    c.mark_word = 0;
    std::vector<NetPass> passes;
    NetGeom g { n, logN, 0 };
#define X(a, b)                                                                                                        \
    if (log_nt == a && log_e == b) {                                                                                   \
        const int lt = a + b;                                                                                          \
        plan_sort(logN, lt, lt - 4 < 8 ? lt - 4 : 8, passes);                                                          \
        return launch_net<R, a, b>(c, g, passes, nullptr, st);                                                         \
    }
    VELO_FOR_REC_TUNES(X)
#undef X
    return einval("velo_osort_records: unsupported tile configuration for records");
}

} // namespace velo

using namespace velo;

extern "C" velo_status velo_osort_records(uint64_t* const* d_words, uint32_t n_words, uint64_t key_mask, size_t n,
                                          size_t capacity, uint32_t flags, const velo_tune* tune, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_words || n_words < 1 || n_words > 3)
        return einval("velo_osort_records: 1..3 words per record");
    for (uint32_t i = 0; i < n_words; i++)
        if (!d_words[i])
            return einval("velo_osort_records: null word array");
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_osort_records: n too large");
    if (capacity < np)
        return einval("velo_osort_records: capacity must be >= next_pow2(n)");
    int log_nt = 8, log_e = 4;
    if (tune && tune->tile_log2) {
        const int nt = ilog2_floor(tune->threads);
        if (tune->threads == 0 || (1u << nt) != tune->threads)
            return einval("velo_tune.threads must be a power of two");
        log_nt = nt;
        log_e = (int)tune->tile_log2 - nt;
    }
    if (np == 1)
        return VELO_OK;
    const bool strict = (flags & VELO_SORT_STRICT) != 0;
    cudaStream_t st = (cudaStream_t)stream;
    switch (n_words * 2 + (strict ? 1 : 0)) {
    case 2:
        return rec_sort<1, false>(d_words, key_mask, n, logN, log_nt, log_e, st);
    case 3:
        return rec_sort<1, true>(d_words, key_mask, n, logN, log_nt, log_e, st);
    case 4:
        return rec_sort<2, false>(d_words, key_mask, n, logN, log_nt, log_e, st);
    case 5:
        return rec_sort<2, true>(d_words, key_mask, n, logN, log_nt, log_e, st);
    case 6:
        return rec_sort<3, false>(d_words, key_mask, n, logN, log_nt, log_e, st);
    default:
        return rec_sort<3, true>(d_words, key_mask, n, logN, log_nt, log_e, st);
    }
}
