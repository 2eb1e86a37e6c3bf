// batch_kv64_split.cu -- multi-table batch kernels for the KV64_SPLIT slot format.
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_kv64_split)
{
    return batch_fmt<FMT_KV64_SPLIT>(a, bucket, lanes, scheme, bk, grid, block, s);
}

}  // namespace pg
