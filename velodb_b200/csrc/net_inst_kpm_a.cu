// Instantiations of the network passes for RowKPM (tile configurations of the autotuner).
#include "net_impl.cuh"

VELO_INSTANTIATE_NET(velo::RowKPM, 8, 3)
VELO_INSTANTIATE_NET(velo::RowKPM, 9, 2)
VELO_INSTANTIATE_NET(velo::RowKPM, 10, 1)
