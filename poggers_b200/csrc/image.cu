// image.cu -- checkpoint images of whole tables (save / restore of resident
// tables).  The reference keeps tables only in device memory; the payload
// here is each level in the reference's own slot layout, so an image's
// levels compare byte for byte with a dump of the reference's table.
#include <stdint.h>
#include <string.h>
#include <cuda_runtime.h>
#include <vector>

#include "poggers_b200.h"
#include "table_internal.h"

namespace {

constexpr char kMagic[8] = {'P', 'G', 'B', '2', 'T', 'B', 'L', '1'};
constexpr uint32_t kVersion = 1;

struct image_header {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    pg_table_config cfg;
    uint64_t seed;
    uint64_t level_bytes[2];
    uint64_t checksum;  // FNV-1a 64 over the payload
    uint8_t reserved[16];
};
static_assert(sizeof(pg_level_config) == 24, "pg_level_config layout");
static_assert(sizeof(pg_table_config) == 64, "pg_table_config layout");
static_assert(sizeof(image_header) == PG_IMAGE_HEADER_BYTES, "image header layout");

// FNV-1a, 64-bit (Fowler, Noll, Vo)
uint64_t fnv1a64(const unsigned char *p, uint64_t n, uint64_t h = 0xcbf29ce484222325ULL)
{
    for (uint64_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}

uint64_t slot_bytes(uint32_t format)
{
    switch (format) {
    case PG_FMT_KV64: return 16;
    case PG_FMT_TAGVAL16:
    case PG_FMT_PACKED_TAGVAL16: return 4;
    default: return 2;  // PG_FMT_TAG16, PG_FMT_PACKED_TAGVAL8
    }
}

uint64_t level_image_bytes(const pg_table_config &c, uint32_t l)
{
    const pg_level_config &L = c.levels[l];
    const uint64_t nb = (L.nslots - 1) / L.bucket_size + 1;
    return nb * L.bucket_size * slot_bytes(c.format);
}

}  // namespace

extern "C" {

uint64_t pg_table_image_bytes(const pg_table *t)
{
    if (!t) return 0;
    uint64_t n = PG_IMAGE_HEADER_BYTES;
    for (uint32_t l = 0; l < t->cfg.nlevels; l++) n += level_image_bytes(t->cfg, l);
    return n;
}

pg_status pg_table_save_image(const pg_table *t, void *host_dst, uint64_t bytes)
{
    if (!t || !host_dst || bytes != pg_table_image_bytes(t)) return PG_ERR_INVALID;
    unsigned char *out = static_cast<unsigned char *>(host_dst);
    image_header h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.header_bytes = PG_IMAGE_HEADER_BYTES;
    h.cfg = t->cfg;
    h.seed = t->desc.lv[0].seed;
    uint64_t off = PG_IMAGE_HEADER_BYTES, sum = 0xcbf29ce484222325ULL;
    for (uint32_t l = 0; l < t->cfg.nlevels; l++) {
        h.level_bytes[l] = level_image_bytes(t->cfg, l);
        pg_status st = pg_table_dump_level(t, l, out + off, h.level_bytes[l]);
        if (st != PG_OK) return st;
        sum = fnv1a64(out + off, h.level_bytes[l], sum);
        off += h.level_bytes[l];
    }
    h.checksum = sum;
    memcpy(out, &h, sizeof(h));
    return PG_OK;
}

pg_status pg_table_load_image(const void *host_src, uint64_t bytes, pg_table **out)
{
    if (!out) return PG_ERR_INVALID;
    *out = nullptr;
    if (!host_src || bytes < PG_IMAGE_HEADER_BYTES) return PG_ERR_INVALID;
    const unsigned char *in = static_cast<const unsigned char *>(host_src);
    image_header h;
    memcpy(&h, in, sizeof(h));
    if (memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion || h.header_bytes != PG_IMAGE_HEADER_BYTES)
        return PG_ERR_INVALID;
    if (h.cfg.nlevels < 1 || h.cfg.nlevels > 2) return PG_ERR_INVALID;
    uint64_t total = PG_IMAGE_HEADER_BYTES, sum = 0xcbf29ce484222325ULL;
    for (uint32_t l = 0; l < h.cfg.nlevels; l++) {
        const pg_level_config &L = h.cfg.levels[l];
        if (L.bucket_size == 0 || L.nslots == 0) return PG_ERR_INVALID;
        if (h.level_bytes[l] != level_image_bytes(h.cfg, l)) return PG_ERR_INVALID;
        if (h.level_bytes[l] > bytes - total) return PG_ERR_INVALID;
        sum = fnv1a64(in + total, h.level_bytes[l], sum);
        total += h.level_bytes[l];
    }
    if (total != bytes || sum != h.checksum) return PG_ERR_INVALID;
    pg_table *t = nullptr;
    pg_status st = pg_table_create(&h.cfg, h.seed, &t);
    if (st != PG_OK) return st;
    uint64_t off = PG_IMAGE_HEADER_BYTES;
    for (uint32_t l = 0; l < h.cfg.nlevels; l++) {
        st = pg_table_load_level(t, l, in + off, h.level_bytes[l]);
        if (st != PG_OK) {
            pg_table_destroy(t);
            return st;
        }
        off += h.level_bytes[l];
    }
    *out = t;
    return PG_OK;
}

}  // extern "C"
