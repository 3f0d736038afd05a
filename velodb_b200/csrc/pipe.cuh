// In-tile merge pass with bulk-copy prefetch (SORT_MERGE passes).
//
// The plain merge kernel loads a tile with per-thread loads, runs the
// phase's in-tile levels and stores it; each CTA waits for its loads, so an
// SM overlaps memory and compute only across its two or three CTAs.  Here one
// persistent CTA per SM loops over tiles with two shared-memory buffers: a
// bulk copy (cp.async.bulk, one per word array, completion counted on an
// mbarrier) brings the next tile into one buffer while the current tile,
// read from the other buffer into registers, runs its levels -- the
// transposes reuse the current buffer -- and is stored from registers.  The
// network, its level order and every address are those of the plain merge
// pass; only the schedule of the loads changes.
//
// Every wait on an mbarrier is bounded by %globaltimer: on expiry the kernel
// records a fault word, waits (bounded) for its other copy in flight and
// returns.  The instrumented trace build keeps the plain merge kernel (its
// loads are the per-thread accesses the trace records).
#pragma once

#include "network.cuh"

namespace velo {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// generic-proxy shared-memory accesses before a later async-proxy write
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\t"
                 "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// bounded wait for phase `parity` of `bar`
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns)
{
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (!mbar_try_wait(bar, parity)) {
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns)
            return false;
    }
    return true;
}

// one bulk copy global -> this CTA's shared memory, counted on `bar`
// (16-byte aligned addresses, a multiple of 16 bytes; no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Staging of one tile per row type: the bulk copies and the read of row r
// from the staged word arrays (row types without one keep the plain merge
// kernel).
template <class R>
struct Stage {
    static constexpr bool ok = false;
};

template <>
struct Stage<RowKP> {
    static constexpr bool ok = true;
    static constexpr size_t bytes(int T) { return (size_t)T * 12; }
    __host__ static bool aligned(const RowKP::Cols& c)
    {
        return ((uintptr_t)c.k % 16) == 0 && ((uintptr_t)c.p % 16) == 0;
    }
    __device__ __forceinline__ static void issue(const RowKP::Cols& c, size_t base, int T, char* buf, uint64_t* bar)
    {
        bulk_g2s(buf, c.k + base, (uint32_t)T * 8, bar);
        bulk_g2s(buf + (size_t)T * 8, c.p + base, (uint32_t)T * 4, bar);
    }
    __device__ __forceinline__ static RowKP read(const char* buf, int T, int r)
    {
        const uint64_t k = reinterpret_cast<const uint64_t*>(buf)[r];
        return RowKP { lo32(k), hi32(k), reinterpret_cast<const uint32_t*>(buf + (size_t)T * 8)[r] };
    }
};

template <int W, int KW, bool S, int KM>
struct Stage<RowRec<W, KW, S, KM>> {
    using R = RowRec<W, KW, S, KM>;
    static constexpr bool ok = true;
    static constexpr size_t bytes(int T) { return (size_t)T * 8 * W; }
    __host__ static bool aligned(const typename R::Cols& c)
    {
        for (int x = 0; x < W; x++)
            if ((uintptr_t)c.w[x] % 16 != 0)
                return false;
        return true;
    }
    __device__ __forceinline__ static void issue(const typename R::Cols& c, size_t base, int T, char* buf,
                                                 uint64_t* bar)
    {
#pragma unroll
        for (int x = 0; x < W; x++)
            bulk_g2s(buf + (size_t)x * T * 8, c.w[x] + base, (uint32_t)T * 8, bar);
    }
    __device__ __forceinline__ static R read(const char* buf, int T, int r)
    {
        R v;
#pragma unroll
        for (int x = 0; x < W; x++)
            v.w[x] = reinterpret_cast<const uint64_t*>(buf + (size_t)x * T * 8)[r];
        return v;
    }
};

// Sorts in 4096-row tiles of 256 threads x 16 rows use the bulk-copy merge
// kernel with the same tile as 512 threads x 8 rows (PIPE_LOG_NT/E): one CTA
// per SM holds both buffers, and 16 warps hide the levels' latency better
// than 8 (the same network, so the same results).
constexpr int PIPE_LOG_NT = 9, PIPE_LOG_E = 3;
template <class R, int LOG_NT, int LOG_E>
constexpr bool pipe_capable()
{
    return LOG_NT == 8 && LOG_E == 4 && Stage<R>::ok;
}

// bytes of one of the two buffers: the staged tile, or the transpose area if
// that is larger
template <class R, int LOG_NT, int LOG_E>
constexpr size_t pipe_buf_bytes()
{
    using N = Net<R, LOG_NT, LOG_E>;
    const size_t a = Stage<R>::bytes(N::T), b = N::smem_rows();
    return ((a > b ? a : b) + 127) & ~(size_t)127;
}

constexpr uint64_t PIPE_WAIT_NS = 2000000000ull;

template <class R, int LOG_NT, int LOG_E>
__global__ void __launch_bounds__(1 << LOG_NT, 1)
    k_merge_pipe(typename R::Cols c, NetGeom g, int K, int ntiles, int* fault)
{
    using N = Net<R, LOG_NT, LOG_E>;
    constexpr int T = N::T, E = N::E, LT = N::LT, S0 = N::S0;
    constexpr size_t BUF = pipe_buf_bytes<R, LOG_NT, LOG_E>();
    constexpr uint32_t TX = (uint32_t)Stage<R>::bytes(T);
    extern __shared__ __align__(128) char sm[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int s_ok;
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    int t = blockIdx.x;
    if (t < ntiles && threadIdx.x == 0) {
        mbar_arrive_expect_tx(&mbar[0], TX);
        Stage<R>::issue(c, (size_t)t << LT, T, sm, &mbar[0]);
    }
    for (int i = 0; t < ntiles; t += gridDim.x, i++) {
        const int cur = i & 1;
        char* buf = sm + (size_t)cur * BUF;
        const int tn = t + gridDim.x;
        if (tn < ntiles && threadIdx.x == 0) {
            // the other buffer held the previous tile's transposes
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&mbar[cur ^ 1], TX);
            Stage<R>::issue(c, (size_t)tn << LT, T, sm + (size_t)(cur ^ 1) * BUF, &mbar[cur ^ 1]);
        }
        // thread 0 waits (bounded) and the CTA decides together, so that no
        // thread leaves while others wait at a barrier
        const uint32_t parity = (uint32_t)(i >> 1) & 1u;
        if (threadIdx.x == 0)
            s_ok = mbar_wait_bounded(&mbar[cur], parity, PIPE_WAIT_NS) ? 1 : 0;
        __syncthreads();
        if (!s_ok) {
            if (threadIdx.x == 0) {
                atomicExch(fault, 1);
                if (tn < ntiles)
                    mbar_wait_bounded(&mbar[cur ^ 1], (uint32_t)((i + 1) >> 1) & 1u, PIPE_WAIT_NS);
            }
            return;
        }
        mbar_try_wait(&mbar[cur], parity); // the completed phase: acquires the copied tile for this thread
        const size_t cta_bits = (size_t)t << LT;
        R v[E];
        const int tp = N::tidpart(S0);
#pragma unroll
        for (int e = 0; e < E; e++)
            v[e] = Stage<R>::read(buf, T, tp | (e << S0));
        // levels LT-1 .. 0 of phase 2^K, direction fixed for the tile (the
        // first transpose's barrier also ends the reads of the staged tile)
        const bool asc_c = ((cta_bits >> K) & 1) == 0;
        int s = S0;
        int b = LT - 1;
        while (b >= 0) {
            if (b < s || b >= s + LOG_E) {
                const int ns = window_down(b, LOG_E, LT);
                N::template transpose<true, true>(v, s, ns, buf);
                s = ns;
            }
            N::bitonic_window(v, c, s, b, s, K, true, asc_c);
            b = s - 1;
        }
        if (s != S0) {
            N::template transpose<true, true>(v, s, S0, buf);
            s = S0;
        }
#pragma unroll
        for (int e = 0; e < E; e++)
            R::store(c, cta_bits | tp | (e << S0), v[e]);
        __syncthreads(); // the buffer is free for the copy two tiles ahead
    }
}

} // namespace velo
