// Instantiations of the network passes for 2-word records (strict=false).
#include "net_impl.cuh"

using RecW2S = velo::RowRec<2, 1, false>;

VELO_INSTANTIATE_NET(RecW2S, 8, 3)
VELO_INSTANTIATE_NET(RecW2S, 9, 3)
VELO_INSTANTIATE_NET(RecW2S, 8, 4)
VELO_INSTANTIATE_NET(RecW2S, 9, 2)
