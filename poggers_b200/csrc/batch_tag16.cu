// batch_tag16.cu -- multi-table batch kernels for the TAG16 slot format.
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_tag16)
{
    return batch_fmt<FMT_TAG16>(a, bucket, lanes, scheme, bk, grid, block, s);
}

}  // namespace pg
