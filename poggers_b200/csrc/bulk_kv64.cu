// bulk_kv64.cu -- bulk kernels instantiated for the KV64 slot format.
#include "bulk_kernels.cuh"

namespace pg {

cudaError_t launch_kv64(int op, uint32_t bucket, uint32_t tile, const table_desc &t, const bulk_args &a, dim3 grid,
                      dim3 block, cudaStream_t s)
{
    return launch_fmt<FMT_KV64>(op, bucket, tile, t, a, grid, block, s);
}

}  // namespace pg
