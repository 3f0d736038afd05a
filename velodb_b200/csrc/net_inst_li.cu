// Instantiations of the network passes for the filter + group-by records:
// 2- and 3-word records ordered on the high 32 bits of word 0.
#include "net_impl.cuh"

using LiRec2 = velo::RowRec<2, 1, false, velo::KEY_HI32>;
using LiRec3 = velo::RowRec<3, 1, false, velo::KEY_HI32>;

VELO_INSTANTIATE_NET(LiRec2, 8, 4)
VELO_INSTANTIATE_NET(LiRec3, 8, 4)
