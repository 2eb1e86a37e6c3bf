// bulk_packed8.cu -- bulk kernels of the bucketed filter with 8-bit tags and values.
#include "bulk_packed.cuh"

namespace pg {

cudaError_t launch_packed8(int op, uint32_t b0, uint32_t b1, uint32_t lanes, const table_desc &t,
                            const packed_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    return launch_packed<8>(op, b0, b1, lanes, t, a, grid, block, s);
}

}  // namespace pg
