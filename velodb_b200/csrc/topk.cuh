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

} // namespace velo
