// Host-side planning and launching of network passes (plain path: one kernel
// launch per pass, stream-ordered).  Included by the .cu files that
// instantiate row types.
#pragma once

#include <vector>

#include "common.hpp"
#include "network.cuh"

namespace velo {

template <class R>
__global__ void __launch_bounds__(256) k_count_marks(typename R::Cols c, size_t n, int LT, uint32_t* counts)
{
    __shared__ uint32_t tmp[33];
    VELO_TRACE_KERNEL(TS_K_COUNT_MARKS);
    count_tile<R>(c, n, LT, blockIdx.x, counts, tmp);
}

__global__ void k_scan_tiles(const uint32_t* counts, int ntiles, uint32_t* prefix, uint64_t* d_count);

// Bitonic pass list for Np = 2^logN rows and tile 2^LT; Lmax fused levels.
inline void plan_sort(int logN, int LT, int Lmax, std::vector<NetPass>& out)
{
    out.push_back(NetPass { P_SORT_TILE, logN < LT ? logN : LT, 0, 0 });
    for (int K = LT + 1; K <= logN; K++) {
        int b = K - 1;
        while (b >= LT) {
            int L = b - LT + 1;
            L = L < Lmax ? L : Lmax;
            out.push_back(NetPass { P_SORT_GLOBAL, K, b, L });
            b -= L;
        }
        out.push_back(NetPass { P_SORT_MERGE, K, 0, 0 });
    }
}

// ORCompact pass list (levels bottom-up).
inline void plan_compact(int logN, int LT, int Lmax, std::vector<NetPass>& out)
{
    out.push_back(NetPass { P_COMPACT_TILE, logN < LT ? logN : LT, 0, 0 });
    int b = LT;
    while (b < logN) {
        int L = logN - b;
        L = L < Lmax ? L : Lmax;
        out.push_back(NetPass { P_COMPACT_GLOBAL, 0, b + L - 1, L });
        b += L;
    }
}

// Largest dynamic shared memory of one CTA on sm_100 (227 KB).
constexpr size_t MAX_SMEM_BYTES = 232448;

// Raises the dynamic shared-memory limit of `kern` once per device; `done`
// must be a static owned by the caller's kernel instantiation.
template <class Kern>
inline velo_status ensure_smem(Kern kern, size_t bytes, int (&done)[64])
{
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev])
        return VELO_OK;
    // static shared memory counts against the same per-CTA limit
    cudaFuncAttributes fa {};
    VELO_CUDA_TRY(cudaFuncGetAttributes(&fa, kern), "cudaFuncGetAttributes");
    const size_t room = MAX_SMEM_BYTES > fa.sharedSizeBytes ? MAX_SMEM_BYTES - fa.sharedSizeBytes : 0;
    VELO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(bytes < room ? bytes : room)),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
    return VELO_OK;
}

// Launches `passes` (all bitonic or all ORCompact kinds) over the tiles; one
// kernel launch per pass.  Defined in net_impl.cuh and explicitly
// instantiated per row type and tile configuration (net_inst_*.cu).
template <class R, int LOG_NT, int LOG_E>
velo_status launch_net(const typename R::Cols& c, const NetGeom& g, const std::vector<NetPass>& passes,
                       const uint32_t* tile_prefix, cudaStream_t st);

// CTA shape of a 4096-row tile (LT = 12) for a RowRec type: 256 threads with
// 16 rows each, or 512 threads with 8 rows each where the W x 16 row words do
// not fit under the 128-register cap of two 256-thread CTAs per SM.  3-word
// sorts with one or two key words keep 16 rows (no spills, and fewer
// transposes: measured faster than 8 rows); 3-word sorts with three key words,
// wider sorts and every 3-word compaction spill at 16 rows.
template <class R>
struct Tile12 {
    static constexpr bool WIDE_SORT = R::WORDS >= 4 || (R::WORDS == 3 && R::KEY_WORDS == 3);
    static constexpr bool WIDE_COMPACT = R::WORDS >= 3;
};

template <class R>
inline velo_status launch_net12(const typename R::Cols& c, const NetGeom& g, const std::vector<NetPass>& passes,
                                const uint32_t* tile_prefix, cudaStream_t st)
{
    const bool compact = !passes.empty() && (passes[0].kind == P_COMPACT_TILE || passes[0].kind == P_COMPACT_GLOBAL);
    if (compact ? Tile12<R>::WIDE_COMPACT : Tile12<R>::WIDE_SORT)
        return launch_net<R, 9, 3>(c, g, passes, tile_prefix, st);
    return launch_net<R, 8, 4>(c, g, passes, tile_prefix, st);
}

// A whole bitonic sort of 2^logN pipeline records in 4096-row tiles (8192-row
// tiles of 512 threads x 16 rows, one global phase fewer, measured 20 %
// slower on 2^23 two-word records).
template <class R>
inline velo_status launch_sort_records(const typename R::Cols& c, int logN, cudaStream_t st)
{
    if (logN <= 0)
        return VELO_OK;
    std::vector<NetPass> passes;
    plan_sort(logN, 12, 8, passes);
    return launch_net12<R>(c, NetGeom { (size_t)1 << logN, logN, 0 }, passes, nullptr, st);
}

template <class R>
inline velo_status launch_count_scan(const typename R::Cols& c, size_t n, int logN, int LT, uint32_t* counts,
                                     uint32_t* prefix, uint64_t* d_count, cudaStream_t st)
{
    const int ntiles = logN > LT ? 1 << (logN - LT) : 1;
    k_count_marks<R><<<ntiles, 256, 0, st>>>(c, n, LT, counts);
    k_scan_tiles<<<1, 1024, 0, st>>>(counts, ntiles, prefix, d_count);
    VELO_CUDA_TRY(cudaGetLastError(), "mark count launch");
    return VELO_OK;
}

// (LOG_NT, LOG_E) pairs compiled for the tunable row types; tile 2^11..2^13
// rows, 256..1024 threads (the autotuner's search space).
#define VELO_FOR_TUNES(X)                                                                                              \
    X(8, 3)                                                                                                            \
    X(9, 2)                                                                                                            \
    X(10, 1)                                                                                                           \
    X(8, 4)                                                                                                            \
    X(9, 3)                                                                                                            \
    X(10, 2)                                                                                                           \
    X(8, 5)                                                                                                            \
    X(9, 4)                                                                                                            \
    X(10, 3)

// the same grid for compaction rows
#define VELO_FOR_TUNES_COMPACT(X)                                                                                      \
    X(8, 3)                                                                                                            \
    X(9, 2)                                                                                                            \
    X(10, 1)                                                                                                           \
    X(8, 4)                                                                                                            \
    X(9, 3)                                                                                                            \
    X(10, 2)                                                                                                           \
    X(8, 5)                                                                                                            \
    X(9, 4)                                                                                                            \
    X(10, 3)

inline bool tune_supported(int log_nt, int log_e)
{
#define X(a, b)                                                                                                        \
    if (log_nt == a && log_e == b)                                                                                     \
        return true;
    VELO_FOR_TUNES(X)
#undef X
    return false;
}

inline velo_status resolve_tune(const velo_tune* tune, int def_log_nt, int def_log_e, int* log_nt, int* log_e)
{
    if (!tune || tune->tile_log2 == 0) {
        *log_nt = def_log_nt;
        *log_e = def_log_e;
        return VELO_OK;
    }
    const int nt = ilog2_floor(tune->threads);
    if (tune->threads == 0 || (1u << nt) != tune->threads)
        return einval("velo_tune.threads must be a power of two");
    const int le = (int)tune->tile_log2 - nt;
    if (!tune_supported(nt, le))
        return einval("unsupported velo_tune (tile_log2, threads) combination");
    *log_nt = nt;
    *log_e = le;
    return VELO_OK;
}

} // namespace velo
