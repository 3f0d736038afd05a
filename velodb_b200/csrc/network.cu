// Plain-path entry points of the two networks for (u64 key, u32 payload)
// rows: velo_osort_kp and velo_ocompact_kpm.
#include <mutex>
#include <atomic>
#include <string>

#include "net_host.cuh"
#include "tma.cuh"

namespace velo {

static thread_local std::string g_last_error;

void set_error(const std::string& msg)
{
    g_last_error = msg;
}

__global__ void k_scan_tiles(const uint32_t* counts, int ntiles, uint32_t* prefix, uint64_t* d_count)
{
    __shared__ uint32_t tmp[33];
    VELO_TRACE_KERNEL(TS_K_SCAN_TILES);
    scan_tiles(counts, ntiles, prefix, d_count, tmp);
}

template <class R>
static velo_status sort_dispatch(const typename R::Cols& c, size_t n, int logN, int log_nt, int log_e,
                                 cudaStream_t st)
{
    std::vector<NetPass> passes;
    NetGeom g { n, logN, 0 };
#define X(a, b)                                                                                                        \
    if (log_nt == a && log_e == b) {                                                                                   \
        const int lt = a + b;                                                                                          \
        plan_sort(logN, lt, lt - 5 < 8 ? lt - 5 : 8, passes);                                                          \
        return launch_net<R, a, b>(c, g, passes, nullptr, st);                                                         \
    }
    VELO_FOR_TUNES(X)
#undef X
    return einval("unsupported tile configuration");
}

template <class R>
static velo_status compact_dispatch(const typename R::Cols& c, size_t n, int logN, int log_nt, int log_e,
                                    uint32_t* counts, uint32_t* prefix, uint64_t* d_count, cudaStream_t st)
{
    std::vector<NetPass> passes;
    NetGeom g { n, logN, 0 };
#define X(a, b)                                                                                                        \
    if (log_nt == a && log_e == b) {                                                                                   \
        const int lt = a + b;                                                                                          \
        velo_status rc = launch_count_scan<R>(c, n, logN, lt, counts, prefix, d_count, st);                            \
        if (rc != VELO_OK)                                                                                             \
            return rc;                                                                                                 \
        plan_compact(logN, lt, lt - 5 < 8 ? lt - 5 : 8, passes);                                                       \
        return launch_net<R, a, b>(c, g, passes, prefix, st);                                                          \
    }
    VELO_FOR_TUNES_COMPACT(X)
#undef X
    return einval("unsupported tile configuration");
}

size_t compact_scratch_for(size_t capacity, int lt)
{
    const int logN = ilog2_floor(next_pow2(capacity));
    const size_t ntiles = logN > lt ? (size_t)1 << (logN - lt) : 1;
    return align_up(ntiles * 4, 256) + align_up((ntiles + 1) * 4, 256);
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_next_pow2(size_t x)
{
    return next_pow2(x);
}

static std::atomic<int> g_stage_timing { 0 };
static thread_local float g_stage_ms[velo::StageTimer::MAX_STAGES];
static thread_local int g_stage_n = 0;

bool velo::stage_timing_on() { return g_stage_timing.load(std::memory_order_relaxed) != 0; }

void velo::store_stage_times(const float* ms, int n)
{
    g_stage_n = n;
    for (int i = 0; i < n; i++)
        g_stage_ms[i] = ms[i];
}

extern "C" void velo_set_stage_timing(int on) { g_stage_timing.store(on ? 1 : 0, std::memory_order_relaxed); }

extern "C" int velo_last_stage_times(float* ms, int capacity)
{
    const int n = capacity < g_stage_n ? capacity : g_stage_n;
    for (int i = 0; ms && i < n; i++)
        ms[i] = g_stage_ms[i];
    return ms ? n : g_stage_n;
}

static std::atomic<int> g_pass_timing { 0 };
constexpr int PASS_LOG_CAP = 1024;
static thread_local velo_pass_time g_pass_log[PASS_LOG_CAP];
static thread_local int g_pass_n = 0;

bool velo::pass_timing_on() { return g_pass_timing.load(std::memory_order_relaxed) != 0; }

void velo::store_pass_time(int kind, int log_n, int row_bytes, float ms)
{
    if (g_pass_n < PASS_LOG_CAP)
        g_pass_log[g_pass_n++] = velo_pass_time { (uint32_t)kind, (uint32_t)log_n, (uint32_t)row_bytes, ms };
}

extern "C" void velo_set_pass_timing(int on)
{
    g_pass_timing.store(on ? 1 : 0, std::memory_order_relaxed);
    g_pass_n = 0;
}

extern "C" void velo_pass_times_clear(void) { g_pass_n = 0; }

static std::atomic<int> g_merge_pipe { 0 };

bool velo::merge_pipe_on() { return g_merge_pipe.load(std::memory_order_relaxed) != 0; }

extern "C" void velo_set_merge_pipeline(int on) { g_merge_pipe.store(on ? 1 : 0, std::memory_order_relaxed); }

static std::atomic<int> g_tensor_tiles { 0 };

bool velo::tensor_tiles_on() { return g_tensor_tiles.load(std::memory_order_relaxed) != 0; }

extern "C" void velo_set_tensor_tile_loads(int on) { g_tensor_tiles.store(on ? 1 : 0, std::memory_order_relaxed); }

static std::mutex g_tma_fault_mu;
static int* g_tma_fault[64] = {};

int* velo::tma_fault_word()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return nullptr;
    std::lock_guard<std::mutex> lk(g_tma_fault_mu);
    if (!g_tma_fault[dev]) {
        int* p = nullptr;
        if (cudaMalloc((void**)&p, sizeof(int)) != cudaSuccess)
            return nullptr;
        if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) {
            cudaFree(p);
            return nullptr;
        }
        g_tma_fault[dev] = p;
    }
    return g_tma_fault[dev];
}

extern "C" int velo_tensor_tile_status(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return -1;
    int* p = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_tma_fault_mu);
        p = g_tma_fault[dev];
    }
    int code = 0;
    if (p && cudaMemcpy(&code, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1;
    return code;
}

namespace {
// cuTensorMapEncodeTiled, taken from the driver through the runtime (no
// link against the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled()
{
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q {};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess
            && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}
} // namespace

bool velo::tma_encode_pass(void* const (&base)[3], const int (&es)[3], int narr, int log_n, int LT, int L, int b_lo,
                           TmaMaps* out)
{
    const EncodeTiled enc = encode_tiled();
    const int C = LT - L;
    if (!enc || narr < 1 || narr > 3 || C < 4 || b_lo < C || b_lo > log_n || L < 0 || L > 8)
        return false;
    const int log_d0 = C < 8 ? C : 8;
    for (int x = 0; x < narr; x++) {
        if (es[x] != 4 && es[x] != 8)
            return false;
        const cuuint64_t dims[3] = { (cuuint64_t)1 << log_d0, (cuuint64_t)1 << (b_lo - log_d0),
                                     (cuuint64_t)1 << (log_n - b_lo) };
        const cuuint64_t strides[2] = { ((cuuint64_t)es[x]) << log_d0, ((cuuint64_t)es[x]) << b_lo };
        const cuuint32_t box[3] = { 1u << log_d0, 1u << (C - log_d0), 1u << L };
        const cuuint32_t estr[3] = { 1, 1, 1 };
        const CUresult r = enc(&out->m[x], es[x] == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                               3, base[x], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return false;
    }
    return true;
}

extern "C" int velo_last_pass_times(velo_pass_time* out, int capacity)
{
    const int n = capacity < g_pass_n ? capacity : g_pass_n;
    for (int i = 0; out && i < n; i++)
        out[i] = g_pass_log[i];
    return out ? n : g_pass_n;
}

extern "C" const char* velo_last_error_text(void)
{
    return g_last_error.c_str();
}

// Default tile of the plain compaction and sort for 2^logN rows: 2048 rows
// (256 threads x 8) up to 2^18 rows, where the passes are latency-bound and
// twice the CTAs finish sooner, 4096 rows (256 x 16) above.  Measured on B200
// (ms of one call, L2 flushed): compaction 2^16 0.060 -> 0.040, 2^18 0.063 ->
// 0.044, 2^20 0.067 -> 0.062, 2^23 0.327 -> 0.282 against 8192-row tiles of
// 512 threads; sort 2^16 0.081 -> 0.060, 2^18 0.105 -> 0.085 against 4096-row
// tiles.
constexpr int DEFAULT_SMALL_LOGN = 18;
static int default_log_e(int logN) { return logN <= DEFAULT_SMALL_LOGN ? 3 : 4; }

extern "C" velo_status velo_osort_kp(uint64_t* d_keys, uint32_t* d_payload, size_t n, size_t capacity,
                                     const velo_tune* tune, void* stream)
{
    if (n == 0)
        return VELO_OK;
    if (!d_keys || !d_payload)
        return einval("velo_osort_kp: null buffer");
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_osort_kp: n too large");
    if (capacity < np)
        return einval("velo_osort_kp: capacity must be >= next_pow2(n)");
    int log_nt, log_e;
    velo_status rc = resolve_tune(tune, 8, default_log_e(logN), &log_nt, &log_e);
    if (rc != VELO_OK)
        return rc;
    if (np == 1)
        return VELO_OK;
    RowKP::Cols c { d_keys, d_payload };
    return sort_dispatch<RowKP>(c, n, logN, log_nt, log_e, (cudaStream_t)stream);
}

extern "C" size_t velo_compact_scratch_bytes(size_t capacity, const velo_tune* tune)
{
    if (tune && tune->tile_log2 != 0) {
        int log_nt = 8, log_e = 4;
        if (resolve_tune(tune, 8, 4, &log_nt, &log_e) != VELO_OK)
            return 0;
        return compact_scratch_for(capacity, log_nt + log_e);
    }
    // the default tiles of any n <= capacity (2048 rows up to 2^18 rows,
    // 4096 above; the persistent command queue's tiles are 4096 rows too)
    const size_t small_cap = (size_t)1 << DEFAULT_SMALL_LOGN;
    const size_t a = compact_scratch_for(capacity < small_cap ? capacity : small_cap, 11);
    const size_t b = compact_scratch_for(capacity, 12);
    return a > b ? a : b;
}

extern "C" velo_status velo_ocompact_kpm(uint64_t* d_keys, uint32_t* d_payload, uint8_t* d_marks, size_t n,
                                         size_t capacity, uint64_t* d_count, void* d_scratch, size_t scratch_bytes,
                                         const velo_tune* tune, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) {
        if (d_count)
            VELO_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st), "cudaMemsetAsync");
        return VELO_OK;
    }
    if (!d_keys || !d_payload || !d_marks)
        return einval("velo_ocompact_kpm: null buffer");
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    if (logN > MAX_LOGN)
        return einval("velo_ocompact_kpm: n too large");
    if (capacity < np)
        return einval("velo_ocompact_kpm: capacity must be >= next_pow2(n)");
    int log_nt, log_e;
    velo_status rc = resolve_tune(tune, 8, default_log_e(logN), &log_nt, &log_e);
    if (rc != VELO_OK)
        return rc;
    const int lt = log_nt + log_e;
    const size_t need = compact_scratch_for(np, lt);
    if (!d_scratch || scratch_bytes < need) {
        set_error("velo_ocompact_kpm: scratch must hold velo_compact_scratch_bytes(capacity) bytes");
        return VELO_ENOMEM;
    }
    const size_t ntiles = logN > lt ? (size_t)1 << (logN - lt) : 1;
    uint32_t* counts = static_cast<uint32_t*>(d_scratch);
    uint32_t* prefix = reinterpret_cast<uint32_t*>(static_cast<char*>(d_scratch) + align_up(ntiles * 4, 256));
    RowKPM::Cols c { d_keys, d_payload, d_marks };
    return compact_dispatch<RowKPM>(c, n, logN, log_nt, log_e, counts, prefix, d_count, st);
}
