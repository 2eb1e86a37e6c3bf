// bulk_tag16.cu -- bulk kernels instantiated for the TAG16 slot format.
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_tag16)
{
    return launch_fmt<FMT_TAG16>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
