// Instantiations of the network passes for RowKP (tile configurations of the autotuner).
#include "net_impl.cuh"

VELO_INSTANTIATE_NET(velo::RowKP, 10, 3)
