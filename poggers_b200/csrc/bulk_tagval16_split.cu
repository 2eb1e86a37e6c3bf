// bulk_tagval16_split.cu -- bulk kernels instantiated for the TAGVAL16_SPLIT slot format.
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_tagval16_split)
{
    return launch_fmt<FMT_TAGVAL16_SPLIT>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
