// bulk_tag16.cu -- bulk kernels instantiated for the TAG16 slot format.
#include "bulk_kernels.cuh"

namespace pg {

cudaError_t launch_tag16(int op, uint32_t bucket, uint32_t tile, const table_desc &t, const bulk_args &a, dim3 grid,
                      dim3 block, cudaStream_t s)
{
    return launch_fmt<FMT_TAG16>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
