// hash.cuh -- hashing, tags and bucket-index arithmetic shared by every
// poggers_b200 table kernel (host and device).
//
// MurmurHash64A of one 8-byte key with a per-hasher seed: the function the
// reference's murmurHasher applies to every key
// (include/poggers/hash_schemes/murmurhash.cuh:20-61, 93-100).  Specialised
// to len == 8 (the table key is always uint64_t), so the tail switch and the
// loop vanish; the result is bit-identical.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__ __forceinline__
#else
#define PG_HD inline
#endif

namespace pg {

constexpr uint64_t kMurmurM = 0xc6a4a7935bd1e995ULL;

PG_HD uint64_t murmur64a_u64(uint64_t key, uint64_t seed)
{
    uint64_t h = seed ^ (8ULL * kMurmurM);
    uint64_t k = key * kMurmurM;
    k ^= k >> 47;
    k *= kMurmurM;
    h ^= k;
    h *= kMurmurM;
    h ^= h >> 47;
    h *= kMurmurM;
    h ^= h >> 47;
    return h;
}

// The 16-bit stored form of a key in the filter formats: the low 16 bits of
// the raw key, with the empty value 0 moved to 1 and the tombstone 0xFFFF
// moved to 0xFFFE (representations/dynamic_container.cuh:35-50).
PG_HD uint16_t tag16(uint64_t key)
{
    uint16_t s = (uint16_t)key;
    s += (s == 0);
    s -= (s == 0xFFFFu);
    return s;
}

PG_HD uint64_t umulhi64(uint64_t a, uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// Remainder by an invariant 64-bit divisor d >= 1, by the round-up method of
// Granlund & Montgomery, "Division by Invariant Integers using
// Multiplication" (PLDI 1994), Fig. 4.1: with l = ceil(log2 d) and
// m = floor(2^64 (2^l - d) / d) + 1,
//   t = mulhi(m, n);  q = (t + ((n - t) >> sh1)) >> sh2,  sh1 = min(l,1), sh2 = max(l-1,0)
// is exact for every 64-bit n.  Replaces the reference's `probe % num_buckets`
// (e.g. insert_schemes/bucket_insert.cuh:137) with one mulhi and one mullo.
struct fastmod64 {
    uint64_t d;
    uint64_t m;
    uint32_t sh1, sh2;

    PG_HD uint64_t mod(uint64_t n) const
    {
        uint64_t t = umulhi64(m, n);
        uint64_t q = (t + ((n - t) >> sh1)) >> sh2;
        return n - q * d;
    }
};

inline fastmod64 make_fastmod64(uint64_t d)
{
    fastmod64 f;
    f.d = d;
    uint32_t l = 0;  // ceil(log2 d)
    while (l < 64 && (((unsigned __int128)1 << l) < d)) l++;
    unsigned __int128 two_l = (unsigned __int128)1 << l;
    unsigned __int128 num = (two_l - d) << 64;
    f.m = (uint64_t)(num / d + 1);
    f.sh1 = l < 1 ? l : 1;
    f.sh2 = l > 0 ? l - 1 : 0;
    return f;
}

// Probing schemes (include/poggers/probing_schemes/):
//   double  h1, h1 + i*h2      double_hashing.cuh:66-95 (hashers seeded s and s*s)
//   linear  h,  h + i          linear_probing.cuh:59-83
//   p2      h1, h2             power_of_two.cuh:68-96   (exactly 2 probes)
//   xor_p2  h1, h1 ^ tag*0x5bd1e995   xor_power_of_two.cuh:64-89 (exactly 2 probes)
// A probe equal to ~0 ends the sequence, like the reference's end() sentinel.
enum probe_kind : uint32_t { PROBE_DOUBLE = 0, PROBE_LINEAR = 1, PROBE_P2 = 2, PROBE_XOR_P2 = 3 };

constexpr uint64_t kProbeEnd = ~0ULL;

struct probe_seq {
    uint64_t h1, h2, key, seed2;
    uint32_t kind;
    bool have2;

    // h1 now; the second hash of double / power-of-two probing only when a
    // probe past the first is asked for (most operations stop at probe 0)
    PG_HD void begin(uint32_t k, uint64_t ky, uint64_t tag, uint64_t seed, uint64_t s2)
    {
        kind = k;
        key = ky;
        seed2 = s2;
        h1 = murmur64a_u64(ky, seed);
        have2 = !(k == PROBE_DOUBLE || k == PROBE_P2);
        h2 = (k == PROBE_XOR_P2) ? (h1 ^ (tag * 0x5bd1e995ULL)) : 1;
    }
    PG_HD uint64_t second()
    {
        if (!have2) {
            h2 = murmur64a_u64(key, seed2);
            have2 = true;
        }
        return h2;
    }
    // raw probe value i (i < max_probes)
    PG_HD uint64_t at(uint32_t i)
    {
        if (i == 0) return h1;
        switch (kind) {
        case PROBE_DOUBLE: return h1 + (uint64_t)i * second();
        case PROBE_LINEAR: return h1 + (uint64_t)i;
        default: return second();  // p2 and xor_p2: the second choice
        }
    }
};

}  // namespace pg
