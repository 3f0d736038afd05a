// Instantiations of the network passes for the pipeline records: the filter +
// group-by records (2 or 3 words ordered on the high 32 bits of word 0) and
// the join union records (2 words ordered on the whole of word 0).
#include "net_impl.cuh"

using LiRec2 = velo::RowRec<2, 1, false, velo::KEY_HI32>;
using LiRec3 = velo::RowRec<3, 1, false, velo::KEY_HI32>;

VELO_INSTANTIATE_NET(LiRec2, 8, 4)
VELO_INSTANTIATE_NET(LiRec3, 8, 4)
VELO_INSTANTIATE_NET(LiRec3, 9, 3)

using JoinRec = velo::RowRec<2, 1, false, velo::KEY_FULL>;
VELO_INSTANTIATE_NET(JoinRec, 8, 4)

// generic group-by records (velo_ogroupby): key word plus 0 or 2 sum words
using GbRec1 = velo::RowRec<1, 1, false, velo::KEY_FULL>;
using GbRec3 = velo::RowRec<3, 1, false, velo::KEY_FULL>;
VELO_INSTANTIATE_NET(GbRec1, 8, 4)
VELO_INSTANTIATE_NET(GbRec3, 8, 4)
VELO_INSTANTIATE_NET(GbRec3, 9, 3)
