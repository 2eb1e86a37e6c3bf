// batch_tagval16_split.cu -- multi-table batch kernels for the TAGVAL16_SPLIT slot format.
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_tagval16_split)
{
    return batch_fmt<FMT_TAGVAL16_SPLIT>(a, bucket, lanes, scheme, bk, grid, block, s);
}

}  // namespace pg
