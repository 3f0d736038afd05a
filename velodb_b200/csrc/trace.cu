// Trace collection entry points (see trace.cuh).  In the product build they
// return VELO_ENOTSUP: only libvelo_obl_trace.so, compiled with -DVELO_TRACE,
// records traces.
#include <cuda_runtime.h>

#include <vector>

#include "common.hpp"
#include "trace.cuh"

#ifdef VELO_TRACE
namespace velo {
namespace trace {
__device__ uint64_t* g_chain = nullptr;
__device__ uint64_t g_slots = 0;
__device__ uint64_t* g_launch = nullptr;
__device__ unsigned long long g_nlaunch = 0;
__device__ uint64_t g_launch_cap = 0;
} // namespace trace
} // namespace velo

static uint64_t* h_chain = nullptr;
static uint64_t* h_launch = nullptr;
static uint64_t h_slots = 0, h_cap = 0;
#endif

using namespace velo;

extern "C" int velo_trace_enabled(void)
{
#ifdef VELO_TRACE
    return 1;
#else
    return 0;
#endif
}

extern "C" velo_status velo_trace_begin(uint64_t slots, uint64_t launch_capacity)
{
#ifdef VELO_TRACE
    if (h_chain)
        return einval("velo_trace_begin: a trace is already open");
    VELO_CUDA_TRY(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    VELO_CUDA_TRY(cudaMalloc(&h_chain, slots * 8), "cudaMalloc(trace chains)");
    VELO_CUDA_TRY(cudaMalloc(&h_launch, launch_capacity * 32), "cudaMalloc(trace launches)");
    VELO_CUDA_TRY(cudaMemset(h_chain, 0, slots * 8), "cudaMemset");
    VELO_CUDA_TRY(cudaMemset(h_launch, 0, launch_capacity * 32), "cudaMemset");
    h_slots = slots;
    h_cap = launch_capacity;
    unsigned long long zero = 0;
    VELO_CUDA_TRY(cudaMemcpyToSymbol(trace::g_chain, &h_chain, sizeof h_chain), "cudaMemcpyToSymbol");
    VELO_CUDA_TRY(cudaMemcpyToSymbol(trace::g_slots, &h_slots, 8), "cudaMemcpyToSymbol");
    VELO_CUDA_TRY(cudaMemcpyToSymbol(trace::g_launch, &h_launch, sizeof h_launch), "cudaMemcpyToSymbol");
    VELO_CUDA_TRY(cudaMemcpyToSymbol(trace::g_nlaunch, &zero, 8), "cudaMemcpyToSymbol");
    VELO_CUDA_TRY(cudaMemcpyToSymbol(trace::g_launch_cap, &h_cap, 8), "cudaMemcpyToSymbol");
    return VELO_OK;
#else
    (void)slots;
    (void)launch_capacity;
    set_error("velo_trace_begin: this library was built without VELO_TRACE");
    return VELO_ENOTSUP;
#endif
}

// Ends the trace: *chain_digest hashes every logical thread's chain in order
// (0 for untouched slots), *touched counts the slots that recorded accesses;
// launches receives up to launch_capacity entries of 4 u64 (kernel id, grid,
// block, dynamic smem) and *n_launches their number.
extern "C" velo_status velo_trace_end(uint64_t* chain_digest, uint64_t* touched, uint64_t* launches,
                                      uint64_t launch_capacity, uint64_t* n_launches)
{
#ifdef VELO_TRACE
    if (!h_chain)
        return einval("velo_trace_end: no open trace");
    VELO_CUDA_TRY(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    std::vector<uint64_t> c(h_slots);
    VELO_CUDA_TRY(cudaMemcpy(c.data(), h_chain, h_slots * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    unsigned long long nl = 0;
    VELO_CUDA_TRY(cudaMemcpyFromSymbol(&nl, trace::g_nlaunch, 8), "cudaMemcpyFromSymbol");
    const uint64_t keep = nl < h_cap ? nl : h_cap;
    std::vector<uint64_t> l(keep * 4);
    if (keep)
        VELO_CUDA_TRY(cudaMemcpy(l.data(), h_launch, keep * 32, cudaMemcpyDeviceToHost), "cudaMemcpy");
    uint64_t d = 0x9E3779B97F4A7C15ull, t = 0;
    for (uint64_t i = 0; i < h_slots; i++) {
        uint64_t z = d ^ (c[i] + 0x632BE59BD9B4E019ull * (i + 1));
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        d = z ^ (z >> 31);
        t += c[i] != 0;
    }
    if (chain_digest)
        *chain_digest = d;
    if (touched)
        *touched = t;
    if (n_launches)
        *n_launches = nl;
    for (uint64_t i = 0; launches && i < keep && i < launch_capacity; i++)
        for (int k = 0; k < 4; k++)
            launches[4 * i + k] = l[4 * i + k];
    uint64_t* null = nullptr;
    uint64_t z = 0;
    cudaMemcpyToSymbol(trace::g_chain, &null, sizeof null);
    cudaMemcpyToSymbol(trace::g_launch, &null, sizeof null);
    cudaMemcpyToSymbol(trace::g_slots, &z, 8);
    cudaFree(h_chain);
    cudaFree(h_launch);
    h_chain = h_launch = nullptr;
    return VELO_OK;
#else
    (void)chain_digest;
    (void)touched;
    (void)launches;
    (void)launch_capacity;
    (void)n_launches;
    set_error("velo_trace_end: this library was built without VELO_TRACE");
    return VELO_ENOTSUP;
#endif
}
