// Definition of launch_net (kernels of the network passes).  Included only by
// the translation units that instantiate it, so each row type / tile
// configuration is compiled once and the instantiations build in parallel.
#pragma once

#include "net_host.cuh"

namespace velo {

// 256-thread CTAs are asked to fit two per SM (at most 128 registers a
// thread): with one 8-warp CTA per SM the in-tile levels stall on latency.
template <int LOG_NT>
constexpr int net_min_blocks() { return LOG_NT <= 8 ? 2 : 1; }

// Passes of one sequence are launched with programmatic stream serialization:
// the next pass may be launched while this one drains, and waits here until
// this pass has completed and its stores are visible, before any global access.
__device__ __forceinline__ void net_pass_prologue()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class R, int LOG_NT, int LOG_E>
__global__ void __launch_bounds__(1 << LOG_NT, net_min_blocks<LOG_NT>())
    k_sort_pass(typename R::Cols c, NetGeom g, NetPass p, const uint32_t* __restrict__ tile_prefix)
{
    extern __shared__ __align__(16) char sm[];
    net_pass_prologue();
    VELO_TRACE_KERNEL(TS_K_SORT_PASS);
    Net<R, LOG_NT, LOG_E>::template run<true>(c, g, p, tile_prefix, blockIdx.x, sm);
}

template <class R, int LOG_NT, int LOG_E>
__global__ void __launch_bounds__(1 << LOG_NT, net_min_blocks<LOG_NT>())
    k_compact_pass(typename R::Cols c, NetGeom g, NetPass p, const uint32_t* __restrict__ tile_prefix)
{
    extern __shared__ __align__(16) char sm[];
    net_pass_prologue();
    VELO_TRACE_KERNEL(TS_K_COMPACT_PASS);
    Net<R, LOG_NT, LOG_E>::template run<false>(c, g, p, tile_prefix, blockIdx.x, sm);
}

template <class R, int LOG_NT, int LOG_E>
velo_status launch_net(const typename R::Cols& c, const NetGeom& g, const std::vector<NetPass>& passes,
                       const uint32_t* tile_prefix, cudaStream_t st)
{
    using N = Net<R, LOG_NT, LOG_E>;
    if (passes.empty())
        return VELO_OK;
    const bool compact = passes[0].kind == P_COMPACT_TILE || passes[0].kind == P_COMPACT_GLOBAL;
    auto kern = compact ? k_compact_pass<R, LOG_NT, LOG_E> : k_sort_pass<R, LOG_NT, LOG_E>;
    const size_t smem = compact ? N::smem_bytes_compact() : N::smem_bytes_sort();
    if (smem > MAX_SMEM_BYTES)
        return einval("tile configuration needs more shared memory than a CTA can have");
    static int done_sort[64] = {}, done_compact[64] = {};
    velo_status rc = ensure_smem(kern, MAX_SMEM_BYTES, compact ? done_compact : done_sort);
    if (rc != VELO_OK)
        return rc;
    const int lt = N::LT;
    const size_t grid = g.logN > lt ? ((size_t)1 << (g.logN - lt)) : 1;
    // the first pass follows whatever ran before it; the later ones overlap
    // their launch with the tail of the previous pass
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    for (size_t i = 0; i < passes.size(); i++) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(1u << LOG_NT);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = i > 0 ? 1 : 0;
        VELO_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, c, g, passes[i], tile_prefix), "network pass launch");
    }
    return VELO_OK;
}

} // namespace velo

#define VELO_INSTANTIATE_NET(R, A, B)                                                                                  \
    template velo_status velo::launch_net<R, A, B>(const typename R::Cols&, const velo::NetGeom&,                      \
                                                   const std::vector<velo::NetPass>&, const uint32_t*, cudaStream_t);
