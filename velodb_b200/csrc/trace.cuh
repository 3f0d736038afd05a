// Address-trace instrumentation (built only with -DVELO_TRACE, into the
// separate test library libvelo_obl_trace.so; the product library compiles
// every macro below to nothing).
//
// Each instrumented global load or store folds (site, address) into a hash
// chain kept per logical thread: logical thread = CTA work index * blockDim +
// threadIdx, where the work index is blockIdx.x for ordinary kernels and the
// claimed item for the persistent scheduler.  Chains continue across the
// launches of one stream.  Block 0 of every instrumented kernel appends
// (kernel id, gridDim, blockDim, dynamic smem bytes) to an ordered launch log.
// An oblivious operator run twice on different data of the same public size,
// through the same buffers, must leave identical chains and launch logs.
#pragma once

#include <cstdint>

#ifdef VELO_TRACE

namespace velo {
namespace trace {

extern __device__ uint64_t* g_chain;
extern __device__ uint64_t g_slots;
extern __device__ uint64_t* g_launch;
extern __device__ unsigned long long g_nlaunch;
extern __device__ uint64_t g_launch_cap;

// work index of the CTA (set at kernel start or per scheduler item)
static __shared__ unsigned long long s_work;

__device__ __forceinline__ uint64_t mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void access(uint32_t site, const void* p)
{
    const uint64_t lid = s_work * blockDim.x + threadIdx.x;
    if (g_chain && lid < g_slots) {
        const uint64_t c = g_chain[lid];
        g_chain[lid] = mix(c ^ mix(((uint64_t)site << 48) ^ (uint64_t)(uintptr_t)p));
    }
}

__device__ __forceinline__ void set_work(unsigned long long w)
{
    __syncthreads();
    if (threadIdx.x == 0)
        s_work = w;
    __syncthreads();
}

__device__ __forceinline__ void kernel_begin(uint32_t site)
{
    set_work(blockIdx.x);
    if (blockIdx.x == 0 && threadIdx.x == 0 && g_launch) {
        uint32_t dsmem;
        asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsmem));
        const unsigned long long i = atomicAdd(&g_nlaunch, 1ull);
        if (i < g_launch_cap) {
            g_launch[4 * i + 0] = site;
            g_launch[4 * i + 1] = gridDim.x;
            g_launch[4 * i + 2] = blockDim.x;
            g_launch[4 * i + 3] = dsmem;
        }
    }
}

} // namespace trace
} // namespace velo

#define VELO_TRACE_KERNEL(site) ::velo::trace::kernel_begin(site)
#define VELO_TRACE_WORK(w) ::velo::trace::set_work(w)
#define VELO_TRACE_AT(site, ptr) ::velo::trace::access(site, (const void*)(ptr))

#else

#define VELO_TRACE_KERNEL(site) ((void)0)
#define VELO_TRACE_WORK(w) ((void)0)
#define VELO_TRACE_AT(site, ptr) ((void)0)

#endif

// launch-log id of a kernel: FNV-1a of its name
constexpr uint32_t velo_site_hash(const char* s, uint32_t h = 2166136261u)
{
    return *s ? velo_site_hash(s + 1, (h ^ (uint32_t)(unsigned char)*s) * 16777619u) : h;
}

// access sites (a site is the code location that issues the access)
enum VeloTraceSite : uint32_t {
    TS_ROW_LOAD = 1,
    TS_ROW_STORE,
    TS_MARK_LOAD,
    TS_TILE_PREFIX,
    TS_TILE_COUNT,
    TS_SCAN,
    TS_K_SORT_PASS = 100,
    TS_K_COMPACT_PASS,
    TS_K_COUNT_MARKS,
    TS_K_SCAN_TILES,
    TS_K_SCHED,
    TS_K_DQ,
    TS_LI_IN = 200,
    TS_LI_OUT,
    TS_SEG_LOAD,
    TS_SEG_META,
    TS_SEG_OUT,
    TS_FILL,
    TS_TOPK,
    TS_GRID, // the index of a grid-stride loop iteration
};

// condition of a grid-stride loop that also records the index visited
#define VELO_GRID_COND(i, n) ((i) < (n) && (VELO_TRACE_AT(TS_GRID, (const void*)(uintptr_t)(i)), true))
