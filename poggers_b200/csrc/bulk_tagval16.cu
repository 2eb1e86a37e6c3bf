// bulk_tagval16.cu -- bulk kernels instantiated for the TAGVAL16 slot format.
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_tagval16)
{
    return launch_fmt<FMT_TAGVAL16>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
