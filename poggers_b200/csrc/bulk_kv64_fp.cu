// bulk_kv64_fp.cu -- bulk kernels for uint64 tables with a fingerprint index
// (one lane per key, bucket_insert primary level; see level_ops_fp).
#include "bulk_kernels.cuh"

namespace pg {

PG_DECLARE_LAUNCH(launch_kv64_fp)
{
    (void)tile;
    const bool bk = t.nlevels > 1;
    switch (bucket) {
    case 4: return bk ? launch_bgs<FMT_KV64_FP, 4, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
                      : launch_bgs<FMT_KV64_FP, 4, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
    case 8: return bk ? launch_bgs<FMT_KV64_FP, 8, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
                      : launch_bgs<FMT_KV64_FP, 8, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
    case 16: return bk ? launch_bgs<FMT_KV64_FP, 16, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
                       : launch_bgs<FMT_KV64_FP, 16, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
    case 32: return bk ? launch_bgs<FMT_KV64_FP, 32, 1, SCHEME_BUCKET, true>(op, t, a, grid, block, s)
                       : launch_bgs<FMT_KV64_FP, 32, 1, SCHEME_BUCKET, false>(op, t, a, grid, block, s);
    default: return cudaErrorInvalidConfiguration;
    }
}

}  // namespace pg
