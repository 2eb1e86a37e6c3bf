// batch_kv64.cu -- multi-table batch kernels for the KV64 slot format.
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_kv64)
{
    return batch_fmt<FMT_KV64>(a, bucket, lanes, scheme, bk, grid, block, s);
}

}  // namespace pg
