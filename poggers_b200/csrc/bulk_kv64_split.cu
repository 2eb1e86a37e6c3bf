// bulk_kv64_split.cu -- bulk kernels instantiated for the KV64_SPLIT slot format.
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_kv64_split)
{
    return launch_fmt<FMT_KV64_SPLIT>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
