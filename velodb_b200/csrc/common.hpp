// Host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "velo_obl.h"

namespace velo {

void set_error(const std::string& msg);

inline velo_status cuda_fail(cudaError_t err, const char* what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return VELO_ECUDA;
}

inline velo_status einval(const std::string& msg)
{
    set_error(msg);
    return VELO_EINVAL;
}

inline int ilog2_floor(size_t x)
{
    int l = -1;
    while (x) {
        l++;
        x >>= 1;
    }
    return l;
}

inline size_t next_pow2(size_t x)
{
    if (x <= 1)
        return 1;
    x--;
    x |= x >> 1;
    x |= x >> 2;
    x |= x >> 4;
    x |= x >> 8;
    x |= x >> 16;
    x |= x >> 32;
    return x + 1;
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Largest supported padded size: the mark prefix counts are u32.
constexpr int MAX_LOGN = 31;

} // namespace velo

#define VELO_CUDA_TRY(call, what)                                                                                      \
    do {                                                                                                               \
        cudaError_t err__ = (call);                                                                                    \
        if (err__ != cudaSuccess)                                                                                      \
            return ::velo::cuda_fail(err__, what);                                                                     \
    } while (0)
