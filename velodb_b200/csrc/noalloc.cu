// velo_ocompact_kpm_noalloc: ORCompact of (key, payload, mark) rows for
// callers that cannot allocate device memory.
//
// Some embedders of this library cannot call cudaMalloc (or any allocating
// routine) at the point where they compact: an engine whose device memory is
// entirely owned by its own pool allocator (an extra cudaMalloc either fails
// once the pool has reserved the HBM or escapes the pool's budget), code on a
// latency-critical path where cudaMalloc's implicit device synchronisation is
// not acceptable, and plugin hosts whose interface offers no allocation hook.
// velo_ocompact_kpm needs a scratch buffer from the caller; this variant
// keeps that scratch in a fixed-size array in the library's own device memory
// instead, so the caller passes only its inputs and outputs.
//
// The array lives for the lifetime of the process on every GPU that loads the
// library (it is a module global), and every call shares it: calls that
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.  Both scratch arrays are fully
// rewritten by every call before they are read (per-tile mark counts, then
// their exclusive prefix), so no state of a previous call can leak into the
// next one and nothing needs clearing.
#include <mutex>

#include "net_host.cuh"

namespace velo {

// Rows per tile of the default configuration (512 threads x 16 rows).
constexpr int NOALLOC_LOG_NT = 9, NOALLOC_LOG_E = 4;
constexpr int NOALLOC_LT = NOALLOC_LOG_NT + NOALLOC_LOG_E;
// Largest supported capacity: 2^28 rows, i.e. 2^15 tiles.
constexpr int NOALLOC_MAX_LOGN = 28;
constexpr size_t NOALLOC_MAX_TILES = (size_t)1 << (NOALLOC_MAX_LOGN - NOALLOC_LT);
// counts[tiles] followed (at a 256-byte boundary) by prefix[tiles + 1]
constexpr size_t NOALLOC_PREFIX_OFFSET = (NOALLOC_MAX_TILES * 4 + 255) / 256 * 256;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_PREFIX_OFFSET + ((NOALLOC_MAX_TILES + 1) * 4 + 255) / 256 * 256;

// The scratch of every call: 131,072 B of counts + 131,328 B of prefix =
// 262,400 B (256 KiB + 256 B).  Host code must not pass this name to a
// kernel: on the host it is only a stand-in for the symbol, so its device
// address is looked up with cudaGetSymbolAddress.
static_assert(NOALLOC_SCRATCH_BYTES == 262400, "the documented size of the no-alloc scratch");
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[64] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this set-up) and kept for the
// life of the process.  A cudaDeviceReset after that first call is not
// supported: the reset rebuilds the module, the array may move, and later
// calls would still use the old address.
static velo_status noalloc_scratch(void** out)
{
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return einval("velo_ocompact_kpm_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess)
            return cuda_fail(err, "cudaGetSymbolAddress(noalloc scratch)");
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" velo_status velo_ocompact_kpm_noalloc(uint64_t* d_keys, uint32_t* d_payload, uint8_t* d_marks, size_t n,
                                                 size_t capacity, uint64_t* d_count, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) {
        if (d_count)
            VELO_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st), "cudaMemsetAsync");
        return VELO_OK;
    }
    if (!d_keys || !d_payload || !d_marks)
        return einval("velo_ocompact_kpm_noalloc: null buffer");
    const size_t np = next_pow2(n);
    if (np > ((size_t)1 << NOALLOC_MAX_LOGN))
        return einval("velo_ocompact_kpm_noalloc: n exceeds the built-in scratch limit of 2^28 rows; "
                      "use velo_ocompact_kpm with a caller-provided scratch buffer");
    if (capacity < np)
        return einval("velo_ocompact_kpm_noalloc: capacity must be >= next_pow2(n)");
    void* scratch = nullptr;
    velo_status rc = noalloc_scratch(&scratch);
    if (rc != VELO_OK)
        return rc;
    const int logN = ilog2_floor(np);
    uint32_t* counts = static_cast<uint32_t*>(scratch);
    uint32_t* prefix = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + NOALLOC_PREFIX_OFFSET);
    RowKPM::Cols c { d_keys, d_payload, d_marks };
    rc = launch_count_scan<RowKPM>(c, n, logN, NOALLOC_LT, counts, prefix, d_count, st);
    if (rc != VELO_OK)
        return rc;
    std::vector<NetPass> passes;
    plan_compact(logN, NOALLOC_LT, NOALLOC_LT - 5 < 8 ? NOALLOC_LT - 5 : 8, passes);
    return launch_net<RowKPM, NOALLOC_LOG_NT, NOALLOC_LOG_E>(c, NetGeom { n, logN, 0 }, passes, prefix, st);
}
