// Instantiations of the network passes for 1-word records (strict=true).
#include "net_impl.cuh"

using RecW1S = velo::RowRec<1, 1, true>;

VELO_INSTANTIATE_NET(RecW1S, 8, 3)
VELO_INSTANTIATE_NET(RecW1S, 9, 3)
VELO_INSTANTIATE_NET(RecW1S, 8, 4)
VELO_INSTANTIATE_NET(RecW1S, 9, 2)
