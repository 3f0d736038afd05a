// Oblivious top-c selection in shared memory (bitonic top-k: sorted runs of c
// rows, merged pairwise keeping the better half).
//
// Rows are two key words (k0, k1) ordered lexicographically on (k0, k1 & m1),
// ascending.  The network is the bitonic sorter's: runs of c rows are sorted
// with alternating directions, so each pair of neighbouring runs is a bitonic
// sequence; the element-wise minimum of such a pair (the half-cleaner's lower
// half) holds its c smallest rows as a bitonic sequence, which c/2 .. 1
// merge levels sort again.  Each round halves the rows until one ascending
// run of c rows, the overall c smallest, is left at the front.  Every
// shared-memory index depends only on (n, c, thread); global memory is not
// touched here.
#pragma once

#include "common.hpp"

namespace velo {

__device__ __forceinline__ bool tk_gt(uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1, uint64_t m1)
{
    const uint64_t x1 = a1 & m1, y1 = b1 & m1;
    return (a0 > b0) | ((a0 == b0) & (x1 > y1));
}

// compare-exchange of rows i < l: ascending puts the smaller row at i
__device__ __forceinline__ void tk_cex(uint64_t* k0, uint64_t* k1, int i, int l, bool asc, uint64_t m1)
{
    const uint64_t a0 = k0[i], a1 = k1[i], b0 = k0[l], b1 = k1[l];
    const bool sw = asc ? tk_gt(a0, a1, b0, b1, m1) : tk_gt(b0, b1, a0, a1, m1);
    k0[i] = sw ? b0 : a0;
    k1[i] = sw ? b1 : a1;
    k0[l] = sw ? a0 : b0;
    k1[l] = sw ? a1 : b1;
}

// index of the p-th pair's lower row at distance j (a zero bit inserted at j)
__device__ __forceinline__ int tk_lower(int p, int j) { return ((p & ~(j - 1)) << 1) | (p & (j - 1)); }

// The c smallest of rows 0..n-1 (powers of two, c <= n <= 2 * P * blockDim.x)
// end up ascending in rows 0..c-1.  With runs_ready the rows already form runs
// of c sorted ascending (even runs) and descending (odd runs).  All threads of
// the block call it; it starts and ends with a barrier.
template <int P>
__device__ void topk_net(uint64_t* k0, uint64_t* k1, int n, int c, uint64_t m1, bool runs_ready)
{
    const int nt = blockDim.x, tid = threadIdx.x;
    int logc = 0;
    while ((1 << logc) < c)
        logc++;
    __syncthreads();
    if (!runs_ready) {
        for (int K = 1; K <= logc; K++) {
            for (int j = 1 << (K - 1); j > 0; j >>= 1) {
                for (int p = tid; p < n / 2; p += nt) {
                    const int i = tk_lower(p, j);
                    tk_cex(k0, k1, i, i | j, ((i >> K) & 1) == 0, m1);
                }
                __syncthreads();
            }
        }
    }
    for (int m = n; m > c; m >>= 1) {
        // lower half of every (ascending, descending) run pair, packed to the
        // front: row p of the result is min(row i, row i + c) of pair p / c
        const int half = m / 2;
        uint64_t r0[P], r1[P];
#pragma unroll
        for (int u = 0; u < P; u++) {
            const int p = tid + u * nt;
            if (p < half) {
                const int i = ((p >> logc) << (logc + 1)) | (p & (c - 1));
                const uint64_t a0 = k0[i], a1 = k1[i], b0 = k0[i + c], b1 = k1[i + c];
                const bool take_b = tk_gt(a0, a1, b0, b1, m1);
                r0[u] = take_b ? b0 : a0;
                r1[u] = take_b ? b1 : a1;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < P; u++) {
            const int p = tid + u * nt;
            if (p < half) {
                k0[p] = r0[u];
                k1[p] = r1[u];
            }
        }
        __syncthreads();
        // each run of c is bitonic: merge it, even runs ascending
        for (int j = c / 2; j > 0; j >>= 1) {
            for (int p = tid; p < half / 2; p += nt) {
                const int i = tk_lower(p, j);
                tk_cex(k0, k1, i, i | j, ((i >> logc) & 1) == 0, m1);
            }
            __syncthreads();
        }
    }
}

// ---- top 16 of a CTA's rows in registers and warp shuffles ------------------
// Lane l of a warp holds rows 4l .. 4l + 3 of the warp's 128 rows (x0[e],
// x1[e] = row 4l + e).  Every exchange partner (register or lane) and every
// direction depends only on the lane and the register, never on the data.

// compare-exchange of registers a (lower row) and b
__device__ __forceinline__ void tk_cx_reg(uint64_t& a0, uint64_t& a1, uint64_t& b0, uint64_t& b1, bool asc,
                                          uint64_t m1)
{
    const bool sw = asc ? tk_gt(a0, a1, b0, b1, m1) : tk_gt(b0, b1, a0, a1, m1);
    const uint64_t n0 = sw ? b0 : a0, n1 = sw ? b1 : a1;
    b0 = sw ? a0 : b0;
    b1 = sw ? a1 : b1;
    a0 = n0;
    a1 = n1;
}

// compare-exchange with lane ^ d: keep the smaller (keep_min) or the larger
// of the two rows; on equal keys each lane keeps its own row
__device__ __forceinline__ void tk_cx_lane(uint64_t& x0, uint64_t& x1, int d, bool keep_min, uint64_t m1)
{
    const uint64_t p0 = __shfl_xor_sync(0xFFFFFFFFu, x0, d), p1 = __shfl_xor_sync(0xFFFFFFFFu, x1, d);
    const bool take = keep_min ? tk_gt(x0, x1, p0, p1, m1) : tk_gt(p0, p1, x0, x1, m1);
    x0 = take ? p0 : x0;
    x1 = take ? p1 : x1;
}

// levels j = 8, 4 (lanes ^ 2, ^ 1) and 2, 1 (registers) of a 16-row run, in
// direction asc
__device__ __forceinline__ void tk_merge16(uint64_t (&x0)[4], uint64_t (&x1)[4], int lane, bool asc, uint64_t m1)
{
#pragma unroll
    for (int d = 2; d >= 1; d >>= 1) {
        const bool lower = (lane & d) == 0;
#pragma unroll
        for (int e = 0; e < 4; e++)
            tk_cx_lane(x0[e], x1[e], d, lower == asc, m1);
    }
    tk_cx_reg(x0[0], x1[0], x0[2], x1[2], asc, m1);
    tk_cx_reg(x0[1], x1[1], x0[3], x1[3], asc, m1);
    tk_cx_reg(x0[0], x1[0], x0[1], x1[1], asc, m1);
    tk_cx_reg(x0[2], x1[2], x0[3], x1[3], asc, m1);
}

// keeps the smaller of row a and row b in a (a on equal keys)
__device__ __forceinline__ void tk_min(uint64_t& a0, uint64_t& a1, uint64_t b0, uint64_t b1, uint64_t m1)
{
    const bool take = tk_gt(a0, a1, b0, b1, m1);
    a0 = take ? b0 : a0;
    a1 = take ? b1 : a1;
}

// Runs of 16 rows (lanes 4q .. 4q + 3 hold run q, row 4(l & 3) + e in
// register e) sorted ascending for even q, descending for odd q, are halved
// three times: the element-wise minimum of a run pair holds its 16 best rows
// as a bitonic sequence, which four merge levels sort again.  Each halving
// keeps only the survivors, so the rows a lane works on halve with the rows:
//   halving 1 (runs q, q ^ 1: lane ^ 4): the lower lane keeps the minima of
//     registers 0 and 1, the upper lane those of registers 2 and 3; the
//     merged run p = l >> 3 is row 4(l & 3) + 2 h + j in register j
//     (h = lane bit 2), merged by lane ^ 2, ^ 1, ^ 4 and the registers;
//   halving 2 (runs p, p ^ 1: lane ^ 8): the lower lane keeps register 0's
//     minimum, the upper register 1's; run l >> 4 is row
//     i(l) = 4(l & 3) + 2((l >> 2) & 1) + ((l >> 3) & 1), one a lane,
//     merged by lane ^ 2, ^ 1, ^ 4, ^ 8;
//   halving 3 (lane ^ 16): both halves keep the minimum and merge ascending.
// On return (r0, r1) of lane l holds row i(l & 15) of the warp's 16 best,
// ascending; lanes l and l ^ 16 hold the same row.  Every partner and
// direction depends only on the lane.
__device__ __forceinline__ void tk_warp_rounds16(const uint64_t (&x0)[4], const uint64_t (&x1)[4], int lane,
                                                 uint64_t m1, uint64_t& r0, uint64_t& r1)
{
    uint64_t a0[2], a1[2];
    {
        const bool h = (lane & 4) != 0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const uint64_t p0 = __shfl_xor_sync(0xFFFFFFFFu, h ? x0[j] : x0[2 + j], 4);
            const uint64_t p1 = __shfl_xor_sync(0xFFFFFFFFu, h ? x1[j] : x1[2 + j], 4);
            a0[j] = h ? x0[2 + j] : x0[j];
            a1[j] = h ? x1[2 + j] : x1[j];
            tk_min(a0[j], a1[j], p0, p1, m1);
        }
        const bool asc = (lane & 8) == 0;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int d = q == 0 ? 2 : q == 1 ? 1 : 4;
            const bool lower = (lane & d) == 0;
#pragma unroll
            for (int j = 0; j < 2; j++)
                tk_cx_lane(a0[j], a1[j], d, lower == asc, m1);
        }
        tk_cx_reg(a0[0], a1[0], a0[1], a1[1], asc, m1);
    }
    {
        const bool h = (lane & 8) != 0;
        const uint64_t p0 = __shfl_xor_sync(0xFFFFFFFFu, h ? a0[0] : a0[1], 8);
        const uint64_t p1 = __shfl_xor_sync(0xFFFFFFFFu, h ? a1[0] : a1[1], 8);
        r0 = h ? a0[1] : a0[0];
        r1 = h ? a1[1] : a1[0];
        tk_min(r0, r1, p0, p1, m1);
        const bool asc = (lane & 16) == 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int d = q == 0 ? 2 : q == 1 ? 1 : q == 2 ? 4 : 8;
            tk_cx_lane(r0, r1, d, ((lane & d) == 0) == asc, m1);
        }
    }
    {
        const uint64_t p0 = __shfl_xor_sync(0xFFFFFFFFu, r0, 16);
        const uint64_t p1 = __shfl_xor_sync(0xFFFFFFFFu, r1, 16);
        tk_min(r0, r1, p0, p1, m1);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int d = q == 0 ? 2 : q == 1 ? 1 : q == 2 ? 4 : 8;
            tk_cx_lane(r0, r1, d, (lane & d) == 0, m1);
        }
    }
}

// row index held by lane l after tk_warp_rounds16
__device__ __forceinline__ int tk_row16(int lane)
{
    return 4 * (lane & 3) + 2 * ((lane >> 2) & 1) + ((lane >> 3) & 1);
}

// Sorts the warp's runs of 16 rows, even runs ascending and odd descending
// (bitonic phases 1..4 of the row index 4 * lane + e).
__device__ __forceinline__ void tk_warp_runs16(uint64_t (&x0)[4], uint64_t (&x1)[4], int lane, uint64_t m1)
{
    // phase 1 (pairs): direction from bit 1 of the row = register bit 1
    tk_cx_reg(x0[0], x1[0], x0[1], x1[1], true, m1);
    tk_cx_reg(x0[2], x1[2], x0[3], x1[3], false, m1);
    // phase 2: direction from bit 2 of the row = lane bit 0
    {
        const bool asc = (lane & 1) == 0;
        tk_cx_reg(x0[0], x1[0], x0[2], x1[2], asc, m1);
        tk_cx_reg(x0[1], x1[1], x0[3], x1[3], asc, m1);
        tk_cx_reg(x0[0], x1[0], x0[1], x1[1], asc, m1);
        tk_cx_reg(x0[2], x1[2], x0[3], x1[3], asc, m1);
    }
    // phase 3: direction from lane bit 1; level 4 across lanes ^ 1
    {
        const bool asc = (lane & 2) == 0;
        const bool lower = (lane & 1) == 0;
#pragma unroll
        for (int e = 0; e < 4; e++)
            tk_cx_lane(x0[e], x1[e], 1, lower == asc, m1);
        tk_cx_reg(x0[0], x1[0], x0[2], x1[2], asc, m1);
        tk_cx_reg(x0[1], x1[1], x0[3], x1[3], asc, m1);
        tk_cx_reg(x0[0], x1[0], x0[1], x1[1], asc, m1);
        tk_cx_reg(x0[2], x1[2], x0[3], x1[3], asc, m1);
    }
    // phase 4: direction from lane bit 2
    tk_merge16(x0, x1, lane, (lane & 4) == 0, m1);
}

// The 16 best of the CTA's rows (4 a thread, blockDim.x = 256): on return
// lane l < 16 of warp 0 holds row tk_row16(l) of them, ascending, in (r0, r1)
// (other threads' values are unspecified).  scratch: 2 x 128 u64 of shared
// memory.
__device__ __forceinline__ void topk16_block(uint64_t (&x0)[4], uint64_t (&x1)[4], uint64_t* scratch, uint64_t m1,
                                             uint64_t& r0, uint64_t& r1)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    tk_warp_runs16(x0, x1, lane, m1);
    tk_warp_rounds16(x0, x1, lane, m1, r0, r1);
    // the 8 warps' results: warp w's 16 rows to rows 16w .. 16w + 15, odd
    // warps reversed so that neighbouring runs form bitonic sequences
    __syncthreads();
    if (lane < 16) {
        const int r = tk_row16(lane);
        const int slot = 16 * warp + ((warp & 1) ? 15 - r : r);
        scratch[slot] = r0;
        scratch[128 + slot] = r1;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            x0[e] = scratch[4 * lane + e];
            x1[e] = scratch[128 + 4 * lane + e];
        }
        tk_warp_rounds16(x0, x1, lane, m1, r0, r1);
    }
}

} // namespace velo
