// slab_pinned.cuh -- the reference's slab policy on sm_100a (device side).
//
// one_size_slab_allocator<extra_blocks> of the reference (include/poggers/
// allocators/slab_one_size.cuh:58-659) pins slabs to SMs and claims objects a
// whole 64-bit word at a time.  This pool keeps that policy, so that its
// results (which calls return NULL, what report_fill says, what the free
// counters count) are the reference's on the same sequence of calls:
//   * slab: a manager word (bit w: word w is whole) over 64 words of 64
//     object bits (bit set: object free) -- offset_alloc_bitarr,
//     offset_slab.cuh:330-675;
//   * per-SM cache: up to 64 entries holding the bits of claimed words that
//     the claiming group did not use -- offset_storage_bitmap, :686-~1110;
//   * per-SM pins: a primary slab and E backups; when the primary has no whole
//     word left it is unpinned, a backup takes its place and the backup's
//     place is refilled from the pool -- smid_pinned_storage, :1466-1780;
//   * pool: slabs neither pinned nor holding objects, one bit each -- the
//     reference's one_size_allocator / veb_tree (one_size_allocator.cuh:43-180);
//   * malloc: at most 25 rounds of cache, then primary, then pivot
//     (slab_one_size.cuh:186-288); free sets the object's bit, completes its
//     word, and returns an emptied unpinned slab to the pool (:428-506).
//
// The mechanics are this library's: a warp's concurrent malloc() calls are
// served together by their leader lane (one claim of a cache entry or a whole
// word, shared out in lane order), so there is no per-warp lock; every loop is
// bounded; random choices come from a hash of the call's position and clock.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace pg {

constexpr uint32_t kPinnedObjects = 4096;
constexpr uint32_t kPinnedMaxAttempts = 25;  // SLAB_ONE_SIZE_MAX_ATTEMPTS (slab_one_size.cuh:20)
constexpr uint32_t kPinnedPlaces = 64;       // pin places per SM (extra_blocks + 1 <= 63)

enum : int { PSLAB_REFUSED = 0, PSLAB_FREED = 1, PSLAB_RETURNED = 2, PSLAB_EMPTIED_PINNED = 3 };

struct pslab_desc {
    unsigned char *pool;             // nslabs * 4096 objects of `size` bytes
    unsigned long long *mgr;         // [nslabs] whole words
    unsigned long long *bits;        // [nslabs * 64] free objects
    unsigned int *pinned;            // [nslabs] 1 = pinned to an SM
    unsigned long long *in_pool;     // [ceil(nslabs / 64)] slab is in the pool
    unsigned long long *cache_claim; // [nsm] free cache entries
    unsigned long long *cache_mgr;   // [nsm] cache entries holding bits
    unsigned long long *cache_bits;  // [nsm * 64]
    unsigned long long *cache_base;  // [nsm * 64] object offset of the entry's word
    long long *pin;                  // [nsm * 64] slab per place, -1 = none; place 0 = primary
    unsigned long long *markers;     // [nsm] live places
    unsigned long long *stats;       // [0] double frees, [1] foreign frees, [2] cache entries lost
    uint64_t size;
    uint64_t nslabs;
    uint32_t nsm;                    // SM ids the per-SM arrays cover (%nsmid)
    uint32_t extra;                  // backups per SM (extra_blocks)
};

__device__ __forceinline__ uint32_t pslab_smid()
{
    uint32_t id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}

__device__ __forceinline__ unsigned long long pslab_ldv(const unsigned long long *p)
{
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

__device__ __forceinline__ uint64_t pslab_hash(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// a pseudo-random set bit of m (m != 0)
__device__ __forceinline__ int pslab_pick(unsigned long long m, uint64_t r)
{
    int k = (int)(r % (uint64_t)__popcll((long long)m));
    for (int i = 0; i < k; ++i) m &= m - 1;
    return __ffsll((long long)m) - 1;
}

// position of the n-th (0-based) set bit of w; w has more than n set bits
__device__ __forceinline__ int pslab_nth(unsigned long long w, int n)
{
    for (int i = 0; i < n; ++i) w &= w - 1;
    return __ffsll((long long)w) - 1;
}

// the n lowest set bits of w (n <= 64)
__device__ __forceinline__ unsigned long long pslab_lowest(unsigned long long w, int n)
{
    unsigned long long m = 0;
    for (int i = 0; i < n && w; ++i) {
        const unsigned long long b = w & (~w + 1);
        m |= b;
        w ^= b;
    }
    return m;
}

// ---- leader-side steps (one lane of the calling group runs each)

// Take one cache entry of SM `sm`: its bits (0 when the cache is empty) and word base.
__device__ __forceinline__ unsigned long long pslab_cache_take(const pslab_desc &S, uint32_t sm, uint64_t r,
                                                               uint64_t &base)
{
    for (int tries = 0; tries < 64; ++tries) {
        const unsigned long long m = pslab_ldv(S.cache_mgr + sm);
        if (!m) return 0ULL;
        const int u = pslab_pick(m, pslab_hash(r + tries));
        const unsigned long long bit = 1ULL << u;
        if (atomicAnd(S.cache_mgr + sm, ~bit) & bit) {
            const unsigned long long bits = atomicExch(S.cache_bits + (uint64_t)sm * 64 + u, 0ULL);
            base = pslab_ldv(S.cache_base + (uint64_t)sm * 64 + u);
            __threadfence();
            atomicOr(S.cache_claim + sm, bit);  // the entry is free again
            return bits;
        }
    }
    return 0ULL;
}

// Put a claimed word's unused bits into a free cache entry (attach_buffer);
// with every entry in use they are lost, as in the reference.
__device__ __forceinline__ void pslab_cache_put(const pslab_desc &S, uint32_t sm, uint64_t r, uint64_t base,
                                                unsigned long long bits)
{
    if (!bits) return;
    for (int tries = 0; tries < 64; ++tries) {
        const unsigned long long c = pslab_ldv(S.cache_claim + sm);
        if (!c) break;
        const int i = pslab_pick(c, pslab_hash(r + 977 * tries));
        const unsigned long long bit = 1ULL << i;
        if (atomicAnd(S.cache_claim + sm, ~bit) & bit) {
            S.cache_base[(uint64_t)sm * 64 + i] = base;
            atomicExch(S.cache_bits + (uint64_t)sm * 64 + i, bits);
            __threadfence();
            atomicOr(S.cache_mgr + sm, bit);
            return;
        }
    }
    atomicAdd(S.stats + 2, 1ULL);
}

// Claim a whole word of slab s (bit_malloc_v2): its bits, or 0 when none is whole.
__device__ __forceinline__ unsigned long long pslab_claim_word(const pslab_desc &S, uint64_t s, uint64_t r, int &w)
{
    for (int tries = 0; tries < 64; ++tries) {
        const unsigned long long m = pslab_ldv(S.mgr + s);
        if (!m) return 0ULL;
        w = pslab_pick(m, pslab_hash(r + 31 * tries));
        const unsigned long long bit = 1ULL << w;
        if (atomicAnd(S.mgr + s, ~bit) & bit) return atomicExch(S.bits + s * 64 + w, 0ULL);
    }
    return 0ULL;
}

// A slab from the pool (a start chosen by r, then the next slab in the pool,
// cyclically), or -1 when the pool is empty.  `lanes` lanes of `mask` look at
// one word each per step.
__device__ __forceinline__ long long pslab_pool_take(const pslab_desc &S, unsigned mask, int rank, int lanes,
                                                     uint64_t r)
{
    const uint64_t nw = (S.nslabs + 63) / 64;
    const uint64_t start = r % nw;
    const uint32_t leader = __ffs(mask) - 1;
    for (uint64_t base = 0; base < nw; base += (uint64_t)lanes) {
        const uint64_t k = base + (uint64_t)rank;
        const uint64_t wi = (start + k) % nw;
        const bool mine = k < nw && pslab_ldv(S.in_pool + wi) != 0ULL;
        unsigned bal = __ballot_sync(mask, mine);
        while (bal) {
            const uint32_t src = __ffs(bal) - 1;
            bal &= bal - 1;
            const uint64_t w = __shfl_sync(mask, wi, src);
            long long got = -1;
            if ((threadIdx.x & 31u) == leader) {
                for (int tries = 0; tries < 64; ++tries) {
                    const unsigned long long m = pslab_ldv(S.in_pool + w);
                    if (!m) break;
                    const int b = __ffsll((long long)m) - 1;
                    if (atomicAnd(S.in_pool + w, ~(1ULL << b)) & (1ULL << b)) {
                        got = (long long)(w * 64 + (uint64_t)b);
                        break;
                    }
                }
            }
            got = __shfl_sync(mask, got, leader);
            if (got >= 0) return got;
        }
    }
    return -1;
}

// pivot_primary (offset_slab.cuh:1513-1578): unpin the primary `prim`, move
// a backup into the primary place; returns the place to refill, or -1 (the
// primary place already taken by another pivot, or no backup left: the
// primary place then stays marked busy and the SM's mallocs fail from now on).
__device__ __forceinline__ int pslab_pivot(const pslab_desc &S, uint32_t sm, long long prim, uint64_t r)
{
    unsigned long long *mk = S.markers + sm;
    if (!(atomicAnd(mk, ~1ULL) & 1ULL)) return -1;
    atomicExch(S.pinned + prim, 0u);
    for (int tries = 0; tries < 64; ++tries) {
        const unsigned long long backups = pslab_ldv(mk) & ~1ULL;
        if (!backups) return -1;
        const int idx = pslab_pick(backups, pslab_hash(r + 613 * tries));
        const unsigned long long bit = 1ULL << idx;
        if (atomicAnd(mk, ~bit) & bit) {
            long long *place = S.pin + (uint64_t)sm * kPinnedPlaces;
            const long long nb = (long long)atomicExch(reinterpret_cast<unsigned long long *>(place + idx),
                                                       (unsigned long long)-1LL);
            if ((long long)atomicCAS(reinterpret_cast<unsigned long long *>(place), (unsigned long long)prim,
                                     (unsigned long long)nb) != prim) {
                // another group replaced the primary meanwhile: put the backup back
                atomicOr(mk, 1ULL);
                if (atomicCAS(reinterpret_cast<unsigned long long *>(place + idx), (unsigned long long)-1LL,
                              (unsigned long long)nb) == (unsigned long long)-1LL)
                    atomicOr(mk, bit);
                return -1;
            }
            atomicOr(mk, 1ULL);
            return idx;
        }
    }
    return -1;
}

// ---- malloc / free

// One malloc() by the lanes of `mask` (every lane of the mask calls it
// together, as slab_malloc's group): each lane gets an object offset, or ~0.
// Per round (at most 25): the SM's cache, then a whole word of the primary
// slab, shared out in lane order, with unused bits cached; lanes still
// unserved then pivot, and the vacated place is refilled from the pool -- when
// the pool is empty the next unserved lane gets NULL (the reference's pivot
// winner) and the rest retry on the new primary.
__device__ __forceinline__ uint64_t pslab_claim(const pslab_desc &S, unsigned mask)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    const int lanes = __popc(mask);
    const uint32_t sm = pslab_smid() % S.nsm;
    long long *place = S.pin + (uint64_t)sm * kPinnedPlaces;
    uint64_t r = 0;
    if (lane == leader) r = pslab_hash((uint64_t)clock64() ^ ((uint64_t)blockIdx.x << 32) ^ threadIdx.x);
    r = __shfl_sync(mask, r, leader);
    uint64_t mine = ~0ULL;
    int served = 0;  // ranks [0, served) are decided: an object, or NULL
    for (uint32_t att = 0; att < kPinnedMaxAttempts && served < lanes; ++att) {
        const uint64_t ra = pslab_hash(r + att);
        long long prim = -1;
        if (lane == leader) prim = (long long)pslab_ldv(reinterpret_cast<const unsigned long long *>(place));
        prim = __shfl_sync(mask, prim, leader);
        if (prim < 0) continue;
        // 1. the SM's cache
        unsigned long long bits = 0;
        uint64_t base = 0;
        if (lane == leader) bits = pslab_cache_take(S, sm, ra, base);
        bits = __shfl_sync(mask, bits, leader);
        base = __shfl_sync(mask, base, leader);
        if (bits) {
            const int c = min(lanes - served, __popcll((long long)bits));
            if (rank >= served && rank < served + c) mine = base + (uint64_t)pslab_nth(bits, rank - served);
            const unsigned long long used = pslab_lowest(bits, c);
            served += c;
            if (served == lanes) {
                if (lane == leader) pslab_cache_put(S, sm, ra + 1, base, bits & ~used);
                break;
            }
        }
        // 2. a whole word of the primary
        int w = 0;
        if (lane == leader) bits = pslab_claim_word(S, (uint64_t)prim, ra + 2, w);
        bits = __shfl_sync(mask, bits, leader);
        w = __shfl_sync(mask, w, leader);
        if (bits) {
            base = (uint64_t)prim * kPinnedObjects + (uint64_t)w * 64;
            const int c = min(lanes - served, __popcll((long long)bits));
            if (rank >= served && rank < served + c) mine = base + (uint64_t)pslab_nth(bits, rank - served);
            const unsigned long long used = pslab_lowest(bits, c);
            served += c;
            if (c > 0 && lane == leader) pslab_cache_put(S, sm, ra + 3, base, bits & ~used);
            if (served == lanes) break;
        }
        // 3. pivot; refill the vacated place from the pool
        int idx = -1;
        if (lane == leader) idx = pslab_pivot(S, sm, prim, ra + 4);
        idx = __shfl_sync(mask, idx, leader);
        if (idx < 0) continue;
        const long long ns = pslab_pool_take(S, mask, rank, lanes, ra + 5);
        if (ns < 0) {
            ++served;  // the pivot's winner returns NULL
            continue;
        }
        for (int q = rank; q < 64; q += lanes) S.bits[(uint64_t)ns * 64 + q] = ~0ULL;
        if (lane == leader) {
            S.mgr[ns] = ~0ULL;
            atomicExch(S.pinned + ns, 1u);
        }
        __threadfence();
        __syncwarp(mask);
        if (lane == leader &&
            atomicCAS(reinterpret_cast<unsigned long long *>(place + idx), (unsigned long long)-1LL,
                      (unsigned long long)ns) == (unsigned long long)-1LL)
            atomicOr(S.markers + sm, 1ULL << idx);
    }
    return mine;
}

// Any thread may call it, from any branch; the group is the lanes that reach
// the call together (see slab_malloc in slab.cuh for why __activemask() is the
// group's mask).
__device__ __forceinline__ void *pslab_malloc(const pslab_desc &S)
{
    const uint64_t off = pslab_claim(S, __activemask());
    return off == ~0ULL ? nullptr : (void *)(S.pool + off * S.size);
}

// free (slab_one_size.cuh:428-463, free_allocation_v2 offset_slab.cuh:455-516):
// PSLAB_REFUSED for a double free (nothing changes; counted in stats[0]) or a
// pointer outside the pool (stats[1]); PSLAB_RETURNED when the free emptied an
// unpinned slab, which goes back to the pool; PSLAB_EMPTIED_PINNED when it
// emptied a pinned one; else PSLAB_FREED.
__device__ __forceinline__ int pslab_release(const pslab_desc &S, const void *p)
{
    const uint64_t byte = (uint64_t)((const unsigned char *)p - S.pool);
    const uint64_t cap = S.nslabs * kPinnedObjects;
    if ((const unsigned char *)p < S.pool || byte % S.size != 0 || byte / S.size >= cap) {
        atomicAdd(S.stats + 1, 1ULL);
        return PSLAB_REFUSED;
    }
    const uint64_t off = byte / S.size;
    const uint64_t s = off / kPinnedObjects;
    const uint32_t w = (uint32_t)((off % kPinnedObjects) / 64);
    const unsigned long long bit = 1ULL << (off % 64);
    const unsigned long long old = atomicOr(S.bits + s * 64 + w, bit);
    if (old & bit) {
        atomicAdd(S.stats, 1ULL);
        return PSLAB_REFUSED;
    }
    if (__popcll((long long)old) != 63) return PSLAB_FREED;
    const unsigned long long om = atomicOr(S.mgr + s, 1ULL << w);
    if ((om & (1ULL << w)) || __popcll((long long)om) != 63) return PSLAB_FREED;
    if (*reinterpret_cast<const volatile unsigned *>(S.pinned + s)) return PSLAB_EMPTIED_PINNED;
    atomicOr(S.in_pool + s / 64, 1ULL << (s % 64));
    return PSLAB_RETURNED;
}

}  // namespace pg
