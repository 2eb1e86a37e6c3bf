// bulk_kv64.cu -- bulk kernels instantiated for the KV64 slot format.
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_kv64)
{
    return launch_fmt<FMT_KV64>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
