/* Host-only stand-in for <cuda.h>, used solely to compile the reference's
 * __host__ __device__ hashing and probing headers with g++ for the oracle
 * pin (oracle/ref_host_pin.cpp).  Defines the CUDA qualifiers away. */
#pragma once
#include <cstddef>
#include <cstdint>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
