// bulk_kv64_fp.cu -- bulk kernels for uint64 tables with a fingerprint index
// (one lane per key, bucket_insert primary level; see level_ops_fp).
#include "bulk_kernels.cuh"

namespace pg {

template <int B>
cudaError_t launch_fp_b(int op, const table_desc &t, const bulk_args &a, dim3 grid, dim3 block, cudaStream_t s)
{
    const bool bk = t.nlevels > 1;
    return bk ? launch_bgs<FMT_KV64_FP, B, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
              : launch_bgs<FMT_KV64_FP, B, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
}

PG_DECLARE_LAUNCH(launch_kv64_fp)
{
    (void)tile;
    switch (bucket) {
    case 4: return launch_fp_b<4>(op, t, a, grid, block, s);
    case 8: return launch_fp_b<8>(op, t, a, grid, block, s);
    case 16: return launch_fp_b<16>(op, t, a, grid, block, s);
    case 32: return launch_fp_b<32>(op, t, a, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

}  // namespace pg
