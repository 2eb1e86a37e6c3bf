// slab.cuh -- fixed-size object allocator (device side).
//
// The reference's one_size_slab_allocator (include/poggers/allocators/
// slab_one_size.cuh:58-659) hands out fixed-size objects from slabs of 4096:
// malloc() returns a distinct pointer into one pool or nullptr after a bounded
// number of attempts (SLAB_ONE_SIZE_MAX_ATTEMPTS = 25, :20), free(ptr) returns
// it, and a double free is detected (offset_slab.cuh:473-478).  Each slab is
// a 64-bit manager word over 64 words of 64 allocation bits
// (offset_slab.cuh:330-675), slabs are pinned per SM (%smid, :1254-1330), and
// a 64-ary bit tree hands out fresh slabs (veb.cuh).
//
// This implementation keeps that geometry and interface and redesigns the
// mechanics for sm_100a:
//   * bits[slab*64 + w]: 1 = object free (4096 per slab);
//   * mgr[slab]: bit w set when word w may hold a free object;
//   * summary[slab/64]: bit set when the slab may hold a free object (the
//     slab-level index that the reference keeps in its vEB tree);
//   * cursor[smid & 255]: the slab each SM allocates from (per-SM pinning);
//   * a warp's concurrent mallocs are served together: its leader claims up
//     to 32 bits of one word with a single atomicAnd and the lanes take them
//     in rank order, so one L2 atomic serves a whole warp;
//   * every loop is bounded; manager and summary bits are hints that a scan
//     repairs, so a lost hint costs a rescan, never an object or a hang.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace pg {

constexpr uint32_t kSlabObjects = 4096;   // objects per slab (64 words x 64 bits)
constexpr uint32_t kSlabWords = 64;
constexpr uint32_t kSlabCursors = 256;    // per-SM cursors, indexed by %smid & 255
// Bounds of one malloc call.  The reference gives up after 25 attempts
// (SLAB_ONE_SIZE_MAX_ATTEMPTS, slab_one_size.cuh:20); here a claim that finds
// nothing because other warps took the bits first, and a move to another slab,
// are bounded separately and more loosely, so that NULL means the pool is full
// rather than contended.  (At 64 idle claims, 75 of 2^22 mallocs over 9 size
// classes with 5 % spare came back NULL: the large classes have few slabs for
// every SM's warps.)
constexpr uint32_t kSlabMaxAttempts = 2048;
constexpr uint32_t kSlabMaxMoves = 1024;

struct slab_desc {
    unsigned char *pool;           // nslabs * 4096 objects of `size` bytes
    unsigned long long *bits;      // nslabs * 64 words, 1 = free
    unsigned long long *mgr;       // nslabs words: word w of the slab may hold a free bit
    unsigned long long *summary;   // ceil(nslabs / 64) words: slab may hold a free object
    unsigned int *cursor;          // kSlabCursors slab ids
    unsigned long long *stats;     // [0] double frees, [1] foreign / misaligned frees
    uint64_t size;                 // object bytes
    uint64_t nslabs;
};

__device__ __forceinline__ uint32_t smid()
{
    uint32_t id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long *p)
{
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

// mask of the lowest k set bits of w (k <= 32)
__device__ __forceinline__ unsigned long long lowest_bits(unsigned long long w, int k)
{
    unsigned long long m = 0;
    for (int i = 0; i < k && w; ++i) {
        unsigned long long b = w & (~w + 1);
        m |= b;
        w ^= b;
    }
    return m;
}

// position of the n-th (0-based) set bit of w; w has more than n set bits
__device__ __forceinline__ int nth_bit(unsigned long long w, int n)
{
    const uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
    const int clo = __popc(lo);
    uint32_t x = n < clo ? lo : hi;
    int base = n < clo ? 0 : 32;
    int r = n < clo ? n : n - clo;
    for (int i = 0; i < r; ++i) x &= x - 1;
    return base + __ffs(x) - 1;
}

// One warp-cooperative malloc: every lane of `mask` calls it together (same
// mask); each gets a distinct object offset, or ~0 once kSlabMaxAttempts
// claims have found nothing, kSlabMaxMoves slab changes were made, or a scan
// of every slab found the pool full.
__device__ __forceinline__ uint64_t slab_claim(const slab_desc &S, unsigned mask)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    const int need = __popc(mask);
    const uint32_t cur_id = smid() & (kSlabCursors - 1);
    // spread the warps of one SM over the words of their slab
    const uint32_t wstart = ((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 37u) & (kSlabWords - 1);
    int assigned = 0;
    uint64_t mine = ~0ULL;
    uint32_t idle = 0, moves = 0;
    for (uint32_t attempt = 0; idle < kSlabMaxAttempts && moves < kSlabMaxMoves && assigned < need; ++attempt) {
        unsigned long long got = 0;
        uint64_t word = 0;
        int state = 0;  // 0 claimed (maybe nothing), 1 slab looks full
        if (lane == leader) {
            const uint32_t slab = __ldcg(S.cursor + cur_id) % (uint32_t)S.nslabs;
            const unsigned long long m = ld_volatile(S.mgr + slab);
            if (m) {
                const unsigned long long rot = (m >> wstart) | (wstart ? (m << (64 - wstart)) : 0ULL);
                const uint32_t wi = (wstart + __ffsll((long long)rot) - 1) & (kSlabWords - 1);
                word = (uint64_t)slab * kSlabWords + wi;
                const unsigned long long snap = ld_volatile(S.bits + word);
                if (snap) {
                    const unsigned long long take = lowest_bits(snap, need - assigned);
                    const unsigned long long old = atomicAnd(S.bits + word, ~take);
                    got = old & take;
                    if ((old & ~take) == 0ULL) {
                        // the word is now empty: drop its manager bit, and the slab's summary bit
                        const unsigned long long om = atomicAnd(S.mgr + slab, ~(1ULL << wi));
                        if (om == (1ULL << wi)) atomicAnd(S.summary + slab / 64, ~(1ULL << (slab % 64)));
                    }
                } else {
                    atomicAnd(S.mgr + slab, ~(1ULL << wi));  // stale hint
                }
            } else {
                state = 1;
                word = slab;
            }
        }
        got = __shfl_sync(mask, got, leader);
        word = __shfl_sync(mask, word, leader);
        state = __shfl_sync(mask, state, leader);
        const int c = __popcll((long long)got);
        if (rank >= assigned && rank < assigned + c) mine = word * 64 + nth_bit(got, rank - assigned);
        assigned += c;
        if (c == 0 && state == 0) ++idle;
        if (state == 1 && assigned < need) {
            ++moves;
            // the pinned slab looks full: repair its manager word from the bits,
            // or move this SM to another slab that the summary lists as free
            const uint32_t slab = (uint32_t)word;
            unsigned long long nz = 0;
            for (uint32_t w = (uint32_t)rank; w < kSlabWords; w += need)
                if (ld_volatile(S.bits + (uint64_t)slab * kSlabWords + w)) nz |= 1ULL << w;
            nz = (unsigned long long)__reduce_or_sync(mask, (unsigned)nz) |
                 ((unsigned long long)__reduce_or_sync(mask, (unsigned)(nz >> 32)) << 32);
            if (nz) {
                if (lane == leader) atomicOr(S.mgr + slab, nz);
                continue;
            }
            uint32_t next = 0xFFFFFFFFu;
            const uint64_t nsum = (S.nslabs + 63) / 64;
            const uint64_t s0 = ((uint64_t)cur_id * 2654435761ULL + attempt * 40503ULL) % nsum;
            for (uint64_t base = 0; base < nsum && next == 0xFFFFFFFFu; base += (uint64_t)need) {
                const uint64_t i = base + (uint64_t)rank;
                unsigned long long sw = 0;
                uint64_t si = 0;
                if (i < nsum) {
                    si = (s0 + i) % nsum;
                    sw = ld_volatile(S.summary + si);
                }
                const unsigned bal = __ballot_sync(mask, sw != 0ULL);
                if (bal) {
                    const uint32_t src = __ffs(bal) - 1;
                    const unsigned long long w = __shfl_sync(mask, sw, src);
                    const uint64_t idx = __shfl_sync(mask, si, src);
                    // a set bit chosen per SM and attempt, so SMs leaving full slabs spread out
                    const uint32_t r = (cur_id * 29u + attempt * 13u) & 63u;
                    const unsigned long long rw = (w >> r) | (r ? (w << (64 - r)) : 0ULL);
                    const uint32_t bit = (r + __ffsll((long long)rw) - 1) & 63u;
                    const uint32_t cand = (uint32_t)(idx * 64 + bit);
                    if (cand < S.nslabs && cand != slab) next = cand;
                    else if (lane == leader) atomicAnd(S.summary + idx, ~(1ULL << bit));
                }
            }
            if (next == 0xFFFFFFFFu) {
                // the summary lists nothing: a bounded scan of every manager word
                // repairs lost summary bits before the pool is declared full
                for (uint64_t base = 0; base < S.nslabs && next == 0xFFFFFFFFu; base += (uint64_t)need) {
                    const uint64_t i = base + (uint64_t)rank;
                    const bool f = i < S.nslabs && i != slab && ld_volatile(S.mgr + i) != 0ULL;
                    const unsigned bal = __ballot_sync(mask, f);
                    if (bal) next = (uint32_t)__shfl_sync(mask, i, __ffs(bal) - 1);
                }
                if (next == 0xFFFFFFFFu) break;  // every slab's manager word is empty: the pool is full
                if (lane == leader) atomicOr(S.summary + next / 64, 1ULL << (next % 64));
            }
            if (lane == leader) atomicCAS(S.cursor + cur_id, slab, next);
        }
    }
    return mine;
}

// Release one object.  Returns false (and counts it) for a pointer outside the
// pool or not on an object boundary, and for a double free.
__device__ __forceinline__ bool slab_release(const slab_desc &S, const void *p)
{
    const uint64_t byte = (uint64_t)((const unsigned char *)p - S.pool);
    const uint64_t cap = S.nslabs * kSlabObjects;
    if ((const unsigned char *)p < S.pool || byte % S.size != 0 || byte / S.size >= cap) {
        atomicAdd(S.stats + 1, 1ULL);
        return false;
    }
    const uint64_t off = byte / S.size;
    const uint64_t slab = off / kSlabObjects;
    const uint32_t w = (uint32_t)((off % kSlabObjects) / 64);
    const unsigned long long bit = 1ULL << (off % 64);
    const unsigned long long old = atomicOr(S.bits + slab * kSlabWords + w, bit);
    if (old & bit) {
        atomicAdd(S.stats, 1ULL);  // double free (offset_slab.cuh:473-478)
        return false;
    }
    if (old == 0ULL) {
        const unsigned long long om = atomicOr(S.mgr + slab, 1ULL << w);
        if (om == 0ULL) atomicOr(S.summary + slab / 64, 1ULL << (slab % 64));
    }
    return true;
}

// Any thread may call it, from any branch (the reference's per-thread
// malloc()).  The lanes of a warp that reach the call together form the group:
// lanes converged at an __activemask() call all receive the same mask, and a
// lane that arrives separately receives a mask without the others.  Every
// warp-synchronizing call in slab_claim names exactly that mask, and its
// control flow is uniform over the group (loop bounds and branches come from
// values broadcast by the leader), so the group's lanes meet at each one.
__device__ __forceinline__ void *slab_malloc(const slab_desc &S)
{
    const uint64_t off = slab_claim(S, __activemask());
    return off == ~0ULL ? nullptr : (void *)(S.pool + off * S.size);
}

}  // namespace pg
