/* poggers_oracle_slabref.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Sequential restatement of the reference's slab allocator,
 * one_size_slab_allocator<extra_blocks> (include/poggers/allocators/
 * slab_one_size.cuh:58-659), with the pieces it is built from:
 *
 *   slab ("offset_alloc_bitarr", offset_slab.cuh:330-675): 4096 objects as a
 *     64-bit manager word over 64 words of 64 allocation bits.  A manager bit
 *     marks a word that is whole (all 64 objects free); a malloc claims a
 *     whole word (manager bit cleared, the word's bits swapped to 0,
 *     bit_malloc_v2 :528-600), and a free sets the object's bit and, when that
 *     completes the word, sets its manager bit again; the free that completes
 *     the last word reports the slab empty (free_allocation_v2 :455-516).
 *   per-SM cache ("offset_storage_bitmap", :686-~1110): the bits of a claimed
 *     word that the calling group did not take, in up to 64 entries; a
 *     malloc takes from it first (bit_malloc_v3), and a word whose entry
 *     cannot be placed (all 64 entries used) is lost.
 *   per-SM pinned slabs ("smid_pinned_storage<E>", :1466-1780): a primary
 *     slab and E backups, taken from the pool when the allocator is created
 *     (init_with_allocators_memory :1710-1748, SMs in order).  When the
 *     primary has no whole word left, pivot_primary (:1513-1578) unpins it,
 *     moves a random backup into the primary place, and the caller refills
 *     the vacated backup place from the pool; with no backup left the pivot
 *     fails and leaves the primary place marked busy, so every later malloc
 *     on that SM fails.
 *   pool ("one_size_allocator" over a veb_tree, one_size_allocator.cuh:43-180):
 *     the slabs that are neither pinned nor holding objects; a take starts at
 *     a random slab and returns the next free one.
 *   malloc (slab_one_size.cuh:186-288): up to SLAB_ONE_SIZE_MAX_ATTEMPTS (25)
 *     rounds of: cache, then primary; on failure one thread of the group wins
 *     the pivot and refills the backup place, returning NULL itself when the
 *     pool is empty; the other threads retry.
 *   free / free_count_misses (:428-506): a double free changes nothing and is
 *     not counted; misses[0] += 1 when the free emptied an unpinned slab (it
 *     goes back to the pool), misses[1] += 1 when it emptied a pinned one.
 *   report_fill / report_max (:628-656): slabs in the pool / slabs in all.
 *
 * The reference's random choices (bits, words, entries, backups, the pool's
 * start) come from a seeded splitmix64 here: which objects a malloc returns
 * differs from any GPU run, as it differs between two runs of the reference;
 * the counts (NULLs, pool size, counters) do not depend on those choices in
 * a sequential run.  Where the reference would attach an invalid slab (more
 * pins at creation than slabs), this model leaves the place empty and counts
 * it in short_pins.
 */
#include <stdlib.h>
#include <string.h>

#include "poggers_oracle.h"

#define RS_OBJECTS 4096
#define RS_MAX_ATTEMPTS 25 /* SLAB_ONE_SIZE_MAX_ATTEMPTS, slab_one_size.cuh:20 */

typedef struct {
    uint64_t manager;   /* bit w: word w is whole and may be claimed */
    uint64_t alloc[64]; /* bit b of word w: object w*64+b is free */
    int pinned;
} rs_slab;

typedef struct {
    uint64_t claim;     /* bit i: entry i is free */
    uint64_t manager;   /* bit i: entry i holds cached bits */
    uint64_t bits[64];
    uint64_t base[64];  /* object offset of the entry's word */
} rs_cache;

typedef struct {
    int64_t ptr[64];    /* slab ids, -1 = empty place; ptr[0] is the primary */
    uint64_t markers;   /* bit i: place i is live */
} rs_pins;

struct pgo_rslab {
    uint64_t nslabs;
    int sms, extra;
    rs_slab *slab;
    uint64_t *pool;     /* bit s: slab s is in the pool */
    uint64_t pool_count;
    rs_cache *cache;
    rs_pins *pins;
    uint64_t rng;
    uint64_t short_pins, lost_words;
};

static uint64_t rs_next(pgo_rslab *a)
{
    uint64_t z = (a->rng += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* a random set bit of m (m != 0) */
static int rs_pick(pgo_rslab *a, uint64_t m)
{
    int k = (int)(rs_next(a) % (uint64_t)__builtin_popcountll(m));
    while (k--) m &= m - 1;
    return __builtin_ctzll(m);
}

static void rs_slab_init(rs_slab *s)
{
    s->manager = ~0ULL;
    for (int w = 0; w < 64; w++) s->alloc[w] = ~0ULL;
    s->pinned = 1;
}

/* the pool's take: a random start, then the next slab in the pool (cyclic) */
static int64_t rs_pool_take(pgo_rslab *a)
{
    if (a->pool_count == 0) return -1;
    const uint64_t start = rs_next(a) % a->nslabs;
    const uint64_t nw = (a->nslabs + 63) / 64;
    for (uint64_t k = 0; k <= nw; k++) {
        const uint64_t wi = (start / 64 + k) % nw;
        uint64_t m = a->pool[wi];
        if (k == 0) m &= ~0ULL << (start % 64);
        if (m) {
            const uint64_t s = wi * 64 + (uint64_t)__builtin_ctzll(m);
            a->pool[wi] &= ~(1ULL << (s % 64));
            a->pool_count--;
            return (int64_t)s;
        }
    }
    return -1; /* not reached: the last pass (k == nw) sees the start word whole */
}

static void rs_pool_put(pgo_rslab *a, uint64_t s)
{
    a->pool[s / 64] |= 1ULL << (s % 64);
    a->pool_count++;
}

/* attach_buffer: the word's leftover bits go to a free cache entry, or are lost */
static void rs_cache_put(pgo_rslab *a, rs_cache *c, uint64_t base, uint64_t bits)
{
    if (!bits) return;
    if (!c->claim) {
        a->lost_words++;
        return;
    }
    const int i = rs_pick(a, c->claim);
    c->claim &= ~(1ULL << i);
    c->base[i] = base;
    c->bits[i] = bits;
    c->manager |= 1ULL << i;
}

pgo_rslab *pgo_rslab_create(uint64_t num_allocs, int sms, int extra_blocks, uint64_t seed)
{
    if (num_allocs == 0 || sms <= 0 || extra_blocks < 0 || extra_blocks > 62) return NULL;
    pgo_rslab *a = (pgo_rslab *)calloc(1, sizeof(pgo_rslab));
    a->nslabs = (num_allocs - 1) / RS_OBJECTS + 1;
    a->sms = sms;
    a->extra = extra_blocks;
    a->rng = seed;
    a->slab = (rs_slab *)calloc(a->nslabs, sizeof(rs_slab));
    a->pool = (uint64_t *)calloc((a->nslabs + 63) / 64, 8);
    for (uint64_t s = 0; s < a->nslabs; s++) rs_pool_put(a, s);
    a->cache = (rs_cache *)calloc((size_t)sms, sizeof(rs_cache));
    a->pins = (rs_pins *)calloc((size_t)sms, sizeof(rs_pins));
    for (int m = 0; m < sms; m++) {
        a->cache[m].claim = ~0ULL;
        for (int i = 0; i < 64; i++) a->pins[m].ptr[i] = -1;
    }
    /* every SM pins a primary and E backups, SMs in order */
    for (int m = 0; m < sms; m++)
        for (int i = 0; i <= extra_blocks; i++) {
            const int64_t s = rs_pool_take(a);
            if (s < 0) {
                a->short_pins++;
                continue;
            }
            rs_slab_init(&a->slab[s]);
            a->pins[m].ptr[i] = s;
            a->pins[m].markers |= 1ULL << i;
        }
    return a;
}

void pgo_rslab_destroy(pgo_rslab *a)
{
    if (!a) return;
    free(a->slab);
    free(a->pool);
    free(a->cache);
    free(a->pins);
    free(a);
}

uint64_t pgo_rslab_report_fill(const pgo_rslab *a) { return a->pool_count; }
uint64_t pgo_rslab_report_max(const pgo_rslab *a) { return a->nslabs; }
uint64_t pgo_rslab_short_pins(const pgo_rslab *a) { return a->short_pins; }
uint64_t pgo_rslab_lost_words(const pgo_rslab *a) { return a->lost_words; }

/* pivot_primary: -1, or the backup place that now needs a slab */
static int rs_pivot(pgo_rslab *a, rs_pins *p, int64_t prim)
{
    if (!(p->markers & 1ULL)) return -1; /* the primary place is already being replaced */
    p->markers &= ~1ULL;
    a->slab[prim].pinned = 0;
    const uint64_t backups = p->markers & ~1ULL;
    if (!backups) return -1; /* no backup: the primary place stays marked busy */
    const int idx = rs_pick(a, backups);
    p->markers &= ~(1ULL << idx);
    p->ptr[0] = p->ptr[idx];
    p->ptr[idx] = -1;
    p->markers |= 1ULL;
    return idx;
}

/* take up to k distinct random bits of *bits into out[0..), object offset base + bit */
static int rs_take(pgo_rslab *a, uint64_t *bits, uint64_t base, int k, uint64_t *out)
{
    int got = 0;
    while (got < k && *bits) {
        const int b = rs_pick(a, *bits);
        *bits &= ~(1ULL << b);
        out[got++] = base + (uint64_t)b;
    }
    return got;
}

uint64_t pgo_rslab_malloc(pgo_rslab *a, int sm, int group, uint64_t *out)
{
    if (!a || sm < 0 || sm >= a->sms || group <= 0 || group > 32) return 0;
    rs_pins *p = &a->pins[sm];
    rs_cache *c = &a->cache[sm];
    uint64_t res[32];
    int done = 0;                       /* threads served, in rank order */
    int pending = group;
    for (int i = 0; i < group; i++) out[i] = ~0ULL;
    for (int att = 0; att < RS_MAX_ATTEMPTS && pending > 0; att++) {
        const int64_t prim = p->ptr[0];
        if (prim < 0) continue;
        /* the SM's cache first */
        if (c->manager) {
            const int u = rs_pick(a, c->manager);
            c->manager &= ~(1ULL << u);
            uint64_t bits = c->bits[u];
            const uint64_t base = c->base[u];
            c->bits[u] = 0;
            c->claim |= 1ULL << u;
            const int got = rs_take(a, &bits, base, pending, res + done);
            done += got;
            pending -= got;
            if (pending == 0) {
                rs_cache_put(a, c, base, bits);
                break;
            }
        }
        /* then a whole word of the primary */
        rs_slab *P = &a->slab[prim];
        if (P->manager) {
            const int w = rs_pick(a, P->manager);
            P->manager &= ~(1ULL << w);
            uint64_t bits = P->alloc[w];
            P->alloc[w] = 0;
            const uint64_t base = (uint64_t)prim * RS_OBJECTS + (uint64_t)w * 64;
            const int got = rs_take(a, &bits, base, pending, res + done);
            done += got;
            pending -= got;
            if (got > 0) rs_cache_put(a, c, base, bits);
            if (pending == 0) break;
        }
        /* the rest failed: one of them wins the pivot and refills the backup place */
        const int idx = rs_pivot(a, p, prim);
        if (idx != -1) {
            const int64_t ns = rs_pool_take(a);
            if (ns < 0) {
                pending--; /* the winner returns NULL */
                res[done++] = ~0ULL;
            } else {
                rs_slab_init(&a->slab[ns]);
                p->ptr[idx] = ns;
                p->markers |= 1ULL << idx;
            }
        }
    }
    uint64_t nulls = 0;
    for (int i = 0; i < done; i++) {
        out[i] = res[i];
        nulls += res[i] == ~0ULL;
    }
    return nulls + (uint64_t)pending;
}

int pgo_rslab_free(pgo_rslab *a, uint64_t offset)
{
    const uint64_t s = offset / RS_OBJECTS;
    if (!a || s >= a->nslabs) return PGO_RSLAB_REFUSED;
    rs_slab *S = &a->slab[s];
    const int w = (int)((offset % RS_OBJECTS) / 64);
    const uint64_t bit = 1ULL << (offset % 64);
    const uint64_t old = S->alloc[w];
    if (old & bit) return PGO_RSLAB_REFUSED; /* double free: nothing changes, nothing counted */
    S->alloc[w] |= bit;
    if (__builtin_popcountll(old) != 63) return PGO_RSLAB_FREED;
    S->alloc[w] = ~0ULL;
    const uint64_t om = S->manager;
    S->manager |= 1ULL << w;
    if ((om & (1ULL << w)) || __builtin_popcountll(om) != 63) return PGO_RSLAB_FREED;
    /* the slab is empty */
    if (S->pinned) return PGO_RSLAB_EMPTIED_PINNED;
    rs_pool_put(a, s);
    return PGO_RSLAB_RETURNED;
}
