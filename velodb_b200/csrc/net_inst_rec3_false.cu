// Instantiations of the network passes for 3-word records (strict=false).
#include "net_impl.cuh"

using RecW3S = velo::RowRec<3, 1, false>;

VELO_INSTANTIATE_NET(RecW3S, 8, 3)
VELO_INSTANTIATE_NET(RecW3S, 9, 3)
VELO_INSTANTIATE_NET(RecW3S, 8, 4)
VELO_INSTANTIATE_NET(RecW3S, 9, 2)
