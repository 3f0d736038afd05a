// Device memory and stream helpers of the C ABI, so that host code above it
// (the C++ operator layer) needs no CUDA headers or runtime of its own.
#include <cuda_runtime.h>

#include "common.hpp"

using namespace velo;

extern "C" velo_status velo_device_alloc(size_t bytes, void* stream, void** out)
{
    if (!out)
        return einval("velo_device_alloc: null argument");
    *out = nullptr;
    if (bytes == 0)
        return VELO_OK;
    const cudaError_t e = cudaMallocAsync(out, bytes, (cudaStream_t)stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        set_error("velo_device_alloc: out of device memory");
        return VELO_ENOMEM;
    }
    VELO_CUDA_TRY(e, "cudaMallocAsync");
    return VELO_OK;
}

extern "C" velo_status velo_device_free(void* p, void* stream)
{
    if (p)
        VELO_CUDA_TRY(cudaFreeAsync(p, (cudaStream_t)stream), "cudaFreeAsync");
    return VELO_OK;
}

extern "C" velo_status velo_copy(void* dst, const void* src, size_t bytes, uint32_t kind, void* stream)
{
    if (bytes == 0)
        return VELO_OK;
    if (!dst || !src)
        return einval("velo_copy: null argument");
    cudaMemcpyKind k;
    switch (kind) {
    case VELO_COPY_H2D:
        k = cudaMemcpyHostToDevice;
        break;
    case VELO_COPY_D2H:
        k = cudaMemcpyDeviceToHost;
        break;
    case VELO_COPY_D2D:
        k = cudaMemcpyDeviceToDevice;
        break;
    default:
        return einval("velo_copy: unknown direction");
    }
    VELO_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream), "cudaMemcpyAsync");
    return VELO_OK;
}

extern "C" velo_status velo_memset(void* dst, int value, size_t bytes, void* stream)
{
    if (bytes == 0)
        return VELO_OK;
    if (!dst)
        return einval("velo_memset: null argument");
    VELO_CUDA_TRY(cudaMemsetAsync(dst, value, bytes, (cudaStream_t)stream), "cudaMemsetAsync");
    return VELO_OK;
}

extern "C" velo_status velo_stream_sync(void* stream)
{
    VELO_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream), "cudaStreamSynchronize");
    return VELO_OK;
}
