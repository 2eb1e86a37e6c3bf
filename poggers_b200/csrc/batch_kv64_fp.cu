// batch_kv64_fp.cu -- multi-table batch kernels for fingerprinted uint64 tables
// (one lane per key, bucket_insert primary).
#include "batch_kernels.cuh"

namespace pg {

PG_DECLARE_BATCH(batch_kv64_fp)
{
    (void)lanes;
    (void)scheme;
    switch (bucket) {
    case 4: return bk ? (k_batch<FMT_KV64_FP, 4, 1, SCHEME_BUCKET, true><<<grid, block, 0, s>>>(a), cudaGetLastError())
                      : (k_batch<FMT_KV64_FP, 4, 1, SCHEME_BUCKET, false><<<grid, block, 0, s>>>(a), cudaGetLastError());
    case 8: return bk ? (k_batch<FMT_KV64_FP, 8, 1, SCHEME_BUCKET, true><<<grid, block, 0, s>>>(a), cudaGetLastError())
                      : (k_batch<FMT_KV64_FP, 8, 1, SCHEME_BUCKET, false><<<grid, block, 0, s>>>(a), cudaGetLastError());
    case 16: return bk ? (k_batch<FMT_KV64_FP, 16, 1, SCHEME_BUCKET, true><<<grid, block, 0, s>>>(a), cudaGetLastError())
                       : (k_batch<FMT_KV64_FP, 16, 1, SCHEME_BUCKET, false><<<grid, block, 0, s>>>(a), cudaGetLastError());
    case 32: return bk ? (k_batch<FMT_KV64_FP, 32, 1, SCHEME_BUCKET, true><<<grid, block, 0, s>>>(a), cudaGetLastError())
                       : (k_batch<FMT_KV64_FP, 32, 1, SCHEME_BUCKET, false><<<grid, block, 0, s>>>(a), cudaGetLastError());
    default: return cudaErrorInvalidConfiguration;
    }
}

}  // namespace pg
