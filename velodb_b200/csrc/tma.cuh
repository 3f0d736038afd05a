// In-tile merge and fused global passes with tensor-map tile loads
// (velo_set_tensor_tile_loads).
//
// The plain pass kernels load a CTA's rows with per-thread loads.  Here one
// thread issues one 3-D tensor-map copy (cp.async.bulk.tensor, no multicast)
// per word array, counted on an mbarrier, that brings the CTA's rows into
// shared memory in local row order; the threads read them from there into
// registers and the pass goes on as in the plain kernel (same network, same
// grid, same results).  The tensor maps cover this GPU's own arrays only.
//
// A CTA's rows: the low C = LT - L bits of the local row index are
// contiguous rows, its upper L bits are global row bits b_lo .. b_hi (a
// fused global pass of L levels; an in-tile merge is C = LT, L = 0).  Viewed
// as a 3-D array of one word array, (d0, 2^b_lo / d0, N / 2^b_lo) with
// d0 = min(2^C, 256), that is one box (d0, 2^C / d0, 2^L) whose innermost
// coordinate is 0, so every copy starts on a 16-byte boundary.
//
// A tensor copy wants its shared-memory destination on a 128-byte boundary
// and its tensor map on a 64-byte one.  The kernel has no static shared
// memory (its mbarrier and flag sit after the tile area of the dynamic
// shared memory), so the dynamic area starts the CTA's shared window; thread
// 0 still checks both alignments before it issues a copy.  A failed check or
// an mbarrier wait that runs out (bounded by %globaltimer) records a code in
// the fault word (tma_fault_word, velo_tensor_tile_status) and the CTA
// returns without storing.  The instrumented trace build keeps the plain
// kernels.
#pragma once

#include <cuda.h>

#include "pipe.cuh"

namespace velo {

// the word arrays of one row type as tensor-map operands
template <class R>
struct TmaRows {
    static constexpr bool ok = false;
};
template <>
struct TmaRows<RowKP> {
    static constexpr bool ok = true;
    static constexpr int NARR = 2;
    static void arrays(const RowKP::Cols& c, void* (&base)[3], int (&es)[3])
    {
        base[0] = c.k;
        es[0] = 8;
        base[1] = c.p;
        es[1] = 4;
    }
};
template <int W, int KW, bool S, int KM>
struct TmaRows<RowRec<W, KW, S, KM>> {
    static constexpr bool ok = W <= 3;
    static constexpr int NARR = W;
    static void arrays(const typename RowRec<W, KW, S, KM>::Cols& c, void* (&base)[3], int (&es)[3])
    {
        for (int x = 0; x < W && x < 3; x++) {
            base[x] = c.w[x];
            es[x] = 8;
        }
    }
};

// one tensor map per word array (kernel parameter, 64-byte aligned)
struct TmaMaps {
    CUtensorMap m[3];
};

// Encodes the maps of one pass (L fused levels, lowest b_lo; L = 0, b_lo = LT
// for an in-tile merge) over arrays of 2^log_n rows; false if the driver
// entry point is missing or an encode fails.
bool tma_encode_pass(void* const (&base)[3], const int (&es)[3], int narr, int log_n, int LT, int L, int b_lo,
                     TmaMaps* out);
// tensor-map tile loads switched on (velo_set_tensor_tile_loads)
bool tensor_tiles_on();
// the calling device's fault word of the tensor-map pass kernels (allocated
// and cleared on first use; nullptr if that fails)
int* tma_fault_word();
// fault codes
constexpr int TMA_FAULT_WAIT = 1, TMA_FAULT_SMEM_ALIGN = 2, TMA_FAULT_MAP_ALIGN = 3;

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x0, int x1, int x2, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
                 "%4}], [%5];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x0), "r"(x1), "r"(x2), "r"(smem_addr(bar))
                 : "memory");
}

constexpr uint64_t TMA_WAIT_NS = 2000000000ull;

// byte offset of the mbarrier (8 bytes) and the CTA's flag (4 bytes) after
// the tile and transpose area; the kernel's dynamic shared memory is
// tma_smem_bytes()
template <class R, int LOG_NT, int LOG_E>
constexpr size_t tma_tail_off()
{
    using N = Net<R, LOG_NT, LOG_E>;
    const size_t a = N::smem_bytes_sort(), b = Stage<R>::bytes(N::T);
    return ((a > b ? a : b) + 15) & ~(size_t)15;
}
template <class R, int LOG_NT, int LOG_E>
constexpr size_t tma_smem_bytes()
{
    return tma_tail_off<R, LOG_NT, LOG_E>() + 16;
}

// WIDE: the three-CTA register budget of the plain kernel of the same shape
template <class R, int LOG_NT, int LOG_E, int PK, int MB, bool WIDE>
__global__ void __launch_bounds__(1 << LOG_NT, MB)
    k_sort_pass_tma(typename R::Cols c, NetGeom g, NetPass p, const __grid_constant__ TmaMaps maps, int* fault)
{
    using N = Net<R, LOG_NT, LOG_E>;
    constexpr int T = N::T, LT = N::LT, NARR = TmaRows<R>::NARR;
    constexpr uint32_t TX = (uint32_t)Stage<R>::bytes(T);
    extern __shared__ __align__(128) char sm[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + tma_tail_off<R, LOG_NT, LOG_E>());
    int* s_code = reinterpret_cast<int*>(sm + tma_tail_off<R, LOG_NT, LOG_E>() + 8);
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // box coordinates of this CTA (see the header comment)
    const bool global = p.kind == P_SORT_GLOBAL;
    const int L = global ? p.L : 0;
    const int C = LT - L;
    const int b_lo = global ? p.b_hi - p.L + 1 : LT;
    const int lo_bits = b_lo - C;
    const int log_d0 = C < 8 ? C : 8;
    const uint32_t cta = blockIdx.x;
    const int x1 = (int)(((cta & ((1u << lo_bits) - 1u)) << C) >> log_d0);
    const int x2 = (int)((cta >> lo_bits) << L);
    if (threadIdx.x == 0) {
        int code = (smem_addr(sm) & 127u) ? TMA_FAULT_SMEM_ALIGN : 0;
#pragma unroll
        for (int x = 0; x < NARR; x++)
            if (reinterpret_cast<uintptr_t>(&maps.m[x]) & 63u)
                code = TMA_FAULT_MAP_ALIGN;
        if (code == 0) {
            mbar_init(mbar, 1);
            mbar_init_fence();
            mbar_arrive_expect_tx(mbar, TX);
            size_t off = 0;
#pragma unroll
            for (int x = 0; x < NARR; x++) {
                tma_load_3d(sm + off, &maps.m[x], 0, x1, x2, mbar);
                // array x's rows: 4-byte payloads of key-payload rows, else words
                off += (size_t)T * (x == 1 && std::is_same_v<R, RowKP> ? 4 : 8);
            }
            if (!mbar_wait_bounded(mbar, 0, TMA_WAIT_NS))
                code = TMA_FAULT_WAIT;
        }
        *s_code = code;
    }
    __syncthreads();
    const int code = *s_code;
    if (code != 0) {
        if (threadIdx.x == 0 && fault)
            atomicExch(fault, code);
        return;
    }
    mbar_try_wait(mbar, 0); // the completed phase: acquires the copied rows for this thread
    N::template run<true, PK, WIDE, Stage<R>>(c, g, p, nullptr, (int)cta, sm);
}

} // namespace velo
