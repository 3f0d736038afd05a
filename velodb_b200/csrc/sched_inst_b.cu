// Instantiations of the persistent scheduler (autotuner tile configurations).
#include "sched_impl.cuh"

VELO_INSTANTIATE_SCHED(8, 4)
VELO_INSTANTIATE_SCHED(9, 3)
VELO_INSTANTIATE_SCHED(10, 2)
