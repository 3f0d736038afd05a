// Instantiations of the network passes for 3-word records (strict=true).
#include "net_impl.cuh"

using RecW3S = velo::RowRec<3, 1, true>;

VELO_INSTANTIATE_NET(RecW3S, 8, 3)
VELO_INSTANTIATE_NET(RecW3S, 9, 3)
VELO_INSTANTIATE_NET(RecW3S, 8, 4)
VELO_INSTANTIATE_NET(RecW3S, 9, 2)
