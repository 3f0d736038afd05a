// Definition of launch_net (kernels of the network passes).  Included only by
// the translation units that instantiate it, so each row type / tile
// configuration is compiled once and the instantiations build in parallel.
#pragma once

#include "net_host.cuh"
#include "pipe.cuh"
#include "tma.cuh"

namespace velo {

// 256-thread CTAs are asked to fit two per SM (at most 128 registers a
// thread): with one 8-warp CTA per SM the in-tile levels stall on latency.
// Some row types also have a three-CTA form (at most 85 registers) for sorts
// of 2^21 rows and more, whose passes need the third CTA to hide latency;
// below that the two-CTA code is faster (2^20 key-payload sort 0.18 ms
// against 0.22 ms, 2^23 1.65 ms against 1.45 ms).
template <class R, int LOG_NT>
constexpr int net_min_blocks() { return LOG_NT <= 8 ? 2 : 1; }
// rows of at most 12 bytes, and two-word records keyed on 32 bits (the
// group-by's: 2^23-row sort 1.78 -> 1.63 ms), in both the in-tile and the
// global kernels.  Two-word records compared on a whole word (the join's
// union) only in the global kernel and the merge kernel: their tile sort
// needs 128 registers (2^23 union sort: tile 353 -> 390 us at 85), while
// their global passes (56.4 -> 53.2 us a pass) and merges (73.9 -> 71.6 us)
// gain from the third CTA.
template <class R>
struct NetWide {
    static constexpr bool ok = sizeof(R) <= 12;
    static constexpr bool ok_global = ok;
};
template <bool S>
struct NetWide<RowRec<2, 1, S, KEY_HI32>> {
    static constexpr bool ok = true;
    static constexpr bool ok_global = true;
};
template <bool S>
struct NetWide<RowRec<2, 1, S, KEY_FULL>> {
    static constexpr bool ok = false;
    static constexpr bool ok_global = true;
};
template <class R, int LOG_NT>
constexpr bool net_has_wide() { return LOG_NT <= 8 && NetWide<R>::ok; }
template <class R, int LOG_NT>
constexpr bool net_has_wide_global() { return LOG_NT <= 8 && NetWide<R>::ok_global; }
constexpr int NET_WIDE_LOGN = 21; // sorts of 2^21 rows and more take the three-CTA form

// Passes of one sequence are launched with programmatic stream serialization:
// the next pass may be launched while this one drains, and waits here until
// this pass has completed and its stores are visible, before any global access.
__device__ __forceinline__ void net_pass_prologue()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// bitonic passes: the tile sort and in-tile merges (PK_LOCAL; record sorts
// run their merges as PK_MERGE) and the fused global passes (PK_GLOBAL) are
// separate kernels
template <class R, int LOG_NT, int LOG_E, int PK, int MB = net_min_blocks<R, LOG_NT>()>
__global__ void __launch_bounds__(1 << LOG_NT, MB)
    k_sort_pass(typename R::Cols c, NetGeom g, NetPass p, const uint32_t* __restrict__ tile_prefix)
{
    extern __shared__ __align__(16) char sm[];
    net_pass_prologue();
    VELO_TRACE_KERNEL(TS_K_SORT_PASS);
    Net<R, LOG_NT, LOG_E>::template run<true, PK, (MB > net_min_blocks<R, LOG_NT>())>(c, g, p, tile_prefix, blockIdx.x,
                                                                                     sm);
}

// ORCompact passes: PK_LOCAL the tile pass, PK_GLOBAL the fused global passes
template <class R, int LOG_NT, int LOG_E, int PK>
__global__ void __launch_bounds__(1 << LOG_NT, net_min_blocks<R, LOG_NT>())
    k_compact_pass(typename R::Cols c, NetGeom g, NetPass p, const uint32_t* __restrict__ tile_prefix)
{
    extern __shared__ __align__(16) char sm[];
    net_pass_prologue();
    VELO_TRACE_KERNEL(TS_K_COMPACT_PASS);
    Net<R, LOG_NT, LOG_E>::template run<false, PK>(c, g, p, tile_prefix, blockIdx.x, sm);
}

// bytes of one row that a pass reads and writes
template <class R>
struct RowBytes {
    static constexpr int value = R::WORDS * 8;
};
template <>
struct RowBytes<RowKP> {
    static constexpr int value = 12;
};
template <>
struct RowBytes<RowKPM> {
    static constexpr int value = 13;
};

// Events around each pass while pass timing is on (velo_set_pass_timing);
// inert otherwise.
class PassTimer {
public:
    PassTimer(cudaStream_t st, size_t n) : st_(st), on_(pass_timing_on()), ev_(on_ ? n + 1 : 0, nullptr)
    {
        for (auto& e : ev_)
            if (cudaEventCreate(&e) != cudaSuccess)
                on_ = false;
        if (on_)
            cudaEventRecord(ev_[0], st_);
    }
    bool on() const { return on_; }
    void mark(size_t i)
    {
        if (on_)
            cudaEventRecord(ev_[i + 1], st_);
    }
    void finish(const std::vector<NetPass>& passes, int log_n, int row_bytes)
    {
        if (!on_ || cudaEventSynchronize(ev_.back()) != cudaSuccess)
            return;
        for (size_t i = 0; i < passes.size(); i++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]);
            store_pass_time(passes[i].kind, log_n, row_bytes, ms);
        }
    }
    ~PassTimer()
    {
        for (auto e : ev_)
            if (e)
                cudaEventDestroy(e);
    }

private:
    cudaStream_t st_;
    bool on_;
    std::vector<cudaEvent_t> ev_;
};

// fault word of the bulk-copy merge kernels of this translation unit
static __device__ int s_pipe_fault;

// The tensor-map pass kernels exist for this row type and tile shape (4096
// rows or more, so that a fused global pass of up to 8 levels keeps at least
// 16 contiguous rows; not in the instrumented trace build) ...
template <class R, int LOG_NT, int LOG_E>
constexpr bool tma_capable()
{
#ifdef VELO_TRACE
    return false;
#else
    return TmaRows<R>::ok && Stage<R>::ok && LOG_NT + LOG_E >= 12;
#endif
}
// ... and are switched on (velo_set_tensor_tile_loads), and the word arrays
// allow tensor-map copies
template <class R, int LOG_NT, int LOG_E>
inline bool tma_passes_on(const typename R::Cols& c)
{
    if constexpr (!tma_capable<R, LOG_NT, LOG_E>()) {
        return false;
    } else {
        return tensor_tiles_on() && Stage<R>::aligned(c) && tma_smem_bytes<R, LOG_NT, LOG_E>() <= MAX_SMEM_BYTES - 1024;
    }
}

// The bulk-copy merge pass (pipe.cuh) for this row type and tile shape, when
// it is switched on (velo_set_merge_pipeline) and the word arrays allow bulk
// copies; returns the grid (one CTA per SM) or 0 for the plain merge kernel.
template <class R, int LOG_NT, int LOG_E>
inline unsigned merge_pipe_grid(const typename R::Cols& c, size_t ntiles, cudaStream_t)
{
#ifdef VELO_TRACE
    return 0;
#else
    if constexpr (!pipe_capable<R, LOG_NT, LOG_E>()) {
        return 0;
    } else {
        if (!merge_pipe_on() || ntiles < 2 || !Stage<R>::aligned(c))
            return 0;
        static int done[64] = {};
        static int sms_of[64] = {};
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
            return 0;
        constexpr size_t smem = 2 * pipe_buf_bytes<R, PIPE_LOG_NT, PIPE_LOG_E>();
        if (smem > MAX_SMEM_BYTES - 1024)
            return 0;
        if (!done[dev]) {
            if (cudaFuncSetAttribute(k_merge_pipe<R, PIPE_LOG_NT, PIPE_LOG_E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem)
                    != cudaSuccess
                || cudaDeviceGetAttribute(&sms_of[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                return 0;
            done[dev] = 1;
        }
        return (unsigned)(ntiles < (size_t)sms_of[dev] ? ntiles : (size_t)sms_of[dev]);
    }
#endif
}

template <class R, int LOG_NT, int LOG_E>
velo_status launch_net(const typename R::Cols& c, const NetGeom& g, const std::vector<NetPass>& passes,
                       const uint32_t* tile_prefix, cudaStream_t st)
{
    using N = Net<R, LOG_NT, LOG_E>;
    if (passes.empty())
        return VELO_OK;
    const bool compact = passes[0].kind == P_COMPACT_TILE || passes[0].kind == P_COMPACT_GLOBAL;
    constexpr int MB = net_min_blocks<R, LOG_NT>();
    constexpr int MBW = net_has_wide<R, LOG_NT>() ? 3 : MB;
    constexpr int MBG = net_has_wide_global<R, LOG_NT>() ? 3 : MB;
    const bool wide = MBW != MB && g.logN >= NET_WIDE_LOGN;
    const bool wide_g = MBG != MB && g.logN >= NET_WIDE_LOGN;
    auto k_local = wide ? k_sort_pass<R, LOG_NT, LOG_E, N::PK_LOCAL, MBW> : k_sort_pass<R, LOG_NT, LOG_E, N::PK_LOCAL, MB>;
    // record sorts run their in-tile merges as a kernel of their own, compiled
    // without the tile-sort code: join union merges 76.5 -> 73.8 us, group-by
    // merges 65.6 -> 62.1 us; key-payload rows keep the shared kernel (2^24
    // merges 111.1 -> 112.9 us with the split)
    constexpr bool split_merge = !std::is_same_v<R, RowKP>;
    // the merges of records that keep a two-CTA tile sort (compared on a
    // whole word) take the global kernel's three-CTA budget from 2^21 rows:
    // 80 registers, a few spilled, join union merges 73.9 -> 71.6 us
    auto k_merge = !split_merge ? k_local
        : wide                  ? k_sort_pass<R, LOG_NT, LOG_E, N::PK_MERGE, MBW>
        : wide_g                ? k_sort_pass<R, LOG_NT, LOG_E, N::PK_MERGE, MBG>
                                : k_sort_pass<R, LOG_NT, LOG_E, N::PK_MERGE, MB>;
    auto k_global = wide_g ? k_sort_pass<R, LOG_NT, LOG_E, N::PK_GLOBAL, MBG>
                           : k_sort_pass<R, LOG_NT, LOG_E, N::PK_GLOBAL, MB>;
    // ORCompact's tile pass and fused global passes are separate kernels too,
    // each compiled without the other's code: join compaction tile pass
    // 98.3 -> 94.2 us, global passes 69.6 -> 65.0 us
    auto k_comp = k_compact_pass<R, LOG_NT, LOG_E, N::PK_LOCAL>;
    auto k_comp_g = k_compact_pass<R, LOG_NT, LOG_E, N::PK_GLOBAL>;
    const size_t smem = compact ? N::smem_bytes_compact() : N::smem_bytes_sort();
    if (smem > MAX_SMEM_BYTES)
        return einval("tile configuration needs more shared memory than a CTA can have");
    static int done_local[2][64] = {}, done_global[2][64] = {}, done_compact[64] = {};
    velo_status rc = compact ? ensure_smem(k_comp, MAX_SMEM_BYTES, done_compact)
                             : ensure_smem(k_local, MAX_SMEM_BYTES, done_local[wide ? 1 : 0]);
    if (rc == VELO_OK && !compact)
        rc = ensure_smem(k_global, MAX_SMEM_BYTES, done_global[wide_g ? 1 : 0]);
    static int done_compact_g[64] = {};
    if (rc == VELO_OK && compact)
        rc = ensure_smem(k_comp_g, MAX_SMEM_BYTES, done_compact_g);
    static int done_merge[3][64] = {};
    if (rc == VELO_OK && !compact && split_merge)
        rc = ensure_smem(k_merge, MAX_SMEM_BYTES, done_merge[wide ? 1 : wide_g ? 2 : 0]);
    if (rc != VELO_OK)
        return rc;
    const int lt = N::LT;
    const size_t grid = g.logN > lt ? ((size_t)1 << (g.logN - lt)) : 1;
    // the first pass follows whatever ran before it; the later ones overlap
    // their launch with the tail of the previous pass
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    const unsigned pipe_grid = compact ? 0u : merge_pipe_grid<R, LOG_NT, LOG_E>(c, grid, st);
    int* pipe_fault = nullptr;
    if (pipe_grid)
        VELO_CUDA_TRY(cudaGetSymbolAddress((void**)&pipe_fault, s_pipe_fault), "cudaGetSymbolAddress");
    const bool tma = !compact && tma_passes_on<R, LOG_NT, LOG_E>(c);
    int* tma_fault = tma ? tma_fault_word() : nullptr;
    PassTimer timer(st, passes.size());
    for (size_t i = 0; i < passes.size(); i++) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(1u << LOG_NT);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = (i > 0 && !timer.on()) ? 1 : 0;
        if (pipe_grid && passes[i].kind == P_SORT_MERGE) {
            if constexpr (pipe_capable<R, LOG_NT, LOG_E>()) {
                cfg.gridDim = dim3(pipe_grid);
                cfg.blockDim = dim3(1u << PIPE_LOG_NT);
                cfg.dynamicSmemBytes = 2 * pipe_buf_bytes<R, PIPE_LOG_NT, PIPE_LOG_E>();
                VELO_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_merge_pipe<R, PIPE_LOG_NT, PIPE_LOG_E>, c, g, passes[i].K,
                                                 (int)grid, pipe_fault),
                              "network merge pass launch");
            }
        } else if (tma && (passes[i].kind == P_SORT_GLOBAL || passes[i].kind == P_SORT_MERGE)) {
            if constexpr (tma_capable<R, LOG_NT, LOG_E>()) {
                const NetPass& q = passes[i];
                const bool gl = q.kind == P_SORT_GLOBAL;
                TmaMaps maps;
                void* base[3] = {};
                int es[3] = {};
                TmaRows<R>::arrays(c, base, es);
                if (!tma_encode_pass(base, es, TmaRows<R>::NARR, g.logN, lt, gl ? q.L : 0, gl ? q.b_hi - q.L + 1 : lt,
                                     &maps))
                    return einval("tensor map encode failed");
                auto kern = gl ? (wide_g ? k_sort_pass_tma<R, LOG_NT, LOG_E, N::PK_GLOBAL, MBG, true>
                                         : k_sort_pass_tma<R, LOG_NT, LOG_E, N::PK_GLOBAL, MB, false>)
                               : (wide ? k_sort_pass_tma<R, LOG_NT, LOG_E, N::PK_LOCAL, MBW, true>
                                       : k_sort_pass_tma<R, LOG_NT, LOG_E, N::PK_LOCAL, MB, false>);
                static int done_tma[4][64] = {};
                const velo_status er =
                    ensure_smem(kern, MAX_SMEM_BYTES, done_tma[(gl ? 2 : 0) + ((gl ? wide_g : wide) ? 1 : 0)]);
                if (er != VELO_OK)
                    return er;
                cfg.dynamicSmemBytes = tma_smem_bytes<R, LOG_NT, LOG_E>();
                VELO_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, c, g, q, maps, tma_fault), "network pass launch");
            }
        } else {
            auto kern = compact ? (passes[i].kind == P_COMPACT_GLOBAL ? k_comp_g : k_comp)
                : passes[i].kind == P_SORT_GLOBAL ? k_global
                : passes[i].kind == P_SORT_MERGE  ? k_merge
                                                  : k_local;
            VELO_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, c, g, passes[i], tile_prefix), "network pass launch");
        }
        timer.mark(i);
    }
    timer.finish(passes, g.logN, RowBytes<R>::value);
    return VELO_OK;
}

} // namespace velo

#define VELO_INSTANTIATE_NET(R, A, B)                                                                                  \
    template velo_status velo::launch_net<R, A, B>(const typename R::Cols&, const velo::NetGeom&,                      \
                                                   const std::vector<velo::NetPass>&, const uint32_t*, cudaStream_t);
