// bulk_tagval16.cu -- bulk kernels instantiated for the TAGVAL16 slot format.
#include "bulk_kernels.cuh"

namespace pg {

cudaError_t launch_tagval16(int op, uint32_t bucket, uint32_t tile, const table_desc &t, const bulk_args &a, dim3 grid,
                      dim3 block, cudaStream_t s)
{
    return launch_fmt<FMT_TAGVAL16>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
