// batch_tagval16.cu -- multi-table batch kernels for the TAGVAL16 slot format.
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_tagval16)
{
    return batch_fmt<FMT_TAGVAL16>(a, bucket, lanes, scheme, bk, grid, block, s);
}

}  // namespace pg
