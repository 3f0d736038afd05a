// Definition of sched_launch (persistent scheduler launch); instantiated per
// tile configuration in sched_inst_*.cu.
#pragma once

#include "net_host.cuh"
#include "sched.cuh"

namespace velo {

template <int LOG_NT, int LOG_E>
velo_status sched_launch(const SchedArgs& a, int sms, cudaStream_t st)
{
    using S = Sched<LOG_NT, LOG_E>;
    auto kern = k_sched<LOG_NT, LOG_E>;
    static int done[64] = {};
    static int occ[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return einval("device ordinal out of range");
    // the kernel also has a few hundred bytes of static shared memory, so the
    // dynamic limit is set to what the configuration needs, not the maximum
    if (S::SMEM + 1024 > MAX_SMEM_BYTES)
        return einval("persistent scheduler configuration needs more shared memory than a CTA can have");
    velo_status rc = ensure_smem(kern, S::SMEM, done);
    if (rc != VELO_OK)
        return rc;
    // occupancy is looked up once per device (first launch), so launches
    // inside a stream capture make no query calls
    if (occ[dev] == 0) {
        int per = 0;
        VELO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 1 << LOG_NT, S::SMEM),
                      "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        occ[dev] = per > 0 ? per : -1;
    }
    const int per_sm = occ[dev];
    if (per_sm < 1)
        return einval("persistent scheduler does not fit on an SM with this tile configuration");
    uint64_t grid = (uint64_t)per_sm * (uint64_t)sms;
    if (grid > a.total_items)
        grid = a.total_items;
    kern<<<(unsigned)grid, 1 << LOG_NT, S::SMEM, st>>>(a);
    VELO_CUDA_TRY(cudaGetLastError(), "persistent scheduler launch");
    return VELO_OK;
}

} // namespace velo

#define VELO_INSTANTIATE_SCHED(A, B) template velo_status velo::sched_launch<A, B>(const velo::SchedArgs&, int, cudaStream_t);
