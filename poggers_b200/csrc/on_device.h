// on_device.h -- the device rule of the C ABI: each call on a table, batch,
// server or allocator runs with the device it was created on current, and is
// refused (PG_ERR_INVALID, nothing launched) otherwise.
#pragma once
#include <cuda_runtime.h>

inline bool pg_on_device(int dev)
{
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return cur == dev;
}
