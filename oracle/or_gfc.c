/*
 * or_gfc.c -- CPU restatement of the reference GFC float compression.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows GfcEncoding::Encode/Decode (compression/gfc/gfc_encoding.cpp:15-108) and
 * CompressDouble/DecompressDouble + _gfcCompressKernelD/_gfcDecompressKernelD
 * (compression/gfc/gfc_encoding_impl_double.cu:31-303) and their float twins
 * (gfc_encoding_impl_float.cu:25-290).  The reference kernels rely on implicit warp synchrony; this
 * restatement evaluates each 32-value subchunk as the warp would if it ran in lock-step.
 */
#include "or_common.h"

typedef struct {
    int wpb, blocks, warps, unit;
    uint64_t n, npad, per;
} gfc_geom_t;

static int gfc_geom(int dt, uint64_t n, int blocks_in, int wpb_in, gfc_geom_t *g)
{
    g->n = n;
    g->npad = (n + 31) & ~31ull;                                    /* impl_double.cu:156-157 */
    g->unit = dt == OR_DOUBLE ? 17 : 9;                             /* (x+1)/2*17 or *9 */
    if (blocks_in > 0) { g->blocks = blocks_in; g->wpb = wpb_in; }
    else {
        g->wpb = dt == OR_DOUBLE ? 16 : 32;                          /* gfc_encoding.cpp:30-33, 77-80 */
        int sub = dt == OR_DOUBLE ? 64 : 32;
        uint64_t bs = (uint64_t)g->wpb * sub * 32;
        g->blocks = (int)((n + bs - 1) / bs);
    }
    if (g->blocks <= 0 || g->wpb <= 0) return OR_ERR_FORMAT;
    g->warps = g->blocks * g->wpb;
    uint64_t per = (g->npad + g->warps - 1) / g->warps;             /* impl_double.cu:170-172 */
    if (per < 32) per = 32;
    per = (per + 31) & ~31ull;
    g->per = per;
    return OR_OK;
}

static inline uint64_t cut_at(const gfc_geom_t *g, int i) /* cut[i] = min((i+1)*per, npad) */
{
    uint64_t c = (uint64_t)(i + 1) * g->per;
    return c < g->npad ? c : g->npad;
}
static inline uint64_t chunk_begin(const gfc_geom_t *g, int w) { return w ? cut_at(g, w - 1) : 0; }
static inline uint64_t scratch_start(const gfc_geom_t *g, int w) { return (chunk_begin(g, w) + 1) / 2 * g->unit; }

static inline uint64_t load_pad(const uint8_t *in, int es, uint64_t n, uint64_t i)
{
    return i < n ? ld_u(in, es, i) : 0;
}

static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

int or_gfc_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *o0, uint8_t *o1, uint8_t *o2, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = ob[2] = 0; return OR_OK; }
    gfc_geom_t g;
    int r = gfc_geom(dt, n, 0, 0, &g);
    if (r) return r;
    uint64_t total = 0;
    for (int w = 0; w < g.warps; w++) {
        uint64_t cb = chunk_begin(&g, w), ce = cut_at(&g, w);
        uint64_t off = scratch_start(&g, w);
        uint64_t last = 0;
        for (uint64_t s = cb; s < ce; s += 32) {
            uint8_t nib[32], mbv[32];
            uint64_t dv[32];
            for (int l = 0; l < 32; l++) {
                uint64_t x = load_pad(in, es, n, s + l), diff;
                int sign, mb, code;
                if (dt == OR_DOUBLE) {
                    diff = x - last;
                    sign = (int)((diff >> 60) & 8);
                    if (sign) diff = 0 - diff;
                    int lz = clz64(diff) >> 3;
                    mb = lz == 6 ? 3 : 8 - lz;
                    code = mb >= 3 ? mb - 1 : mb;
                } else {
                    uint32_t d32 = (uint32_t)x - (uint32_t)last;
                    sign = (int)((d32 >> 28) & 8);
                    if (sign) d32 = 0u - d32;
                    mb = 4 - (clz32(d32) >> 3);
                    code = mb;
                    diff = d32;
                }
                nib[l] = (uint8_t)(sign | code);
                mbv[l] = (uint8_t)mb;
                dv[l] = diff;
            }
            for (int k = 0; k < 16; k++) o2[total++] = (uint8_t)(nib[2 * k] | (nib[2 * k + 1] << 4));
            uint64_t sum = 0;
            for (int l = 0; l < 32; l++)
                for (int b = 0; b < mbv[l]; b++) { o2[total++] = (uint8_t)(dv[l] >> (8 * b)); sum++; }
            off += 16 + sum;
            last = load_pad(in, es, n, cb + 31);  /* impl_double.cu:86: constant after subchunk 0 */
        }
        int32_t end = (int32_t)off;
        memcpy(o1 + 4 * (uint64_t)w, &end, 4);
    }
    int32_t meta[3] = {g.blocks, g.wpb, (int32_t)n};
    memcpy(o0, meta, 12);
    ob[0] = 12; ob[1] = 4 * (uint64_t)g.warps; ob[2] = total;
    return OR_OK;
}

int or_gfc_decode(int dt, const uint8_t *i0, uint64_t b0, const uint8_t *i1, uint64_t b1,
                  const uint8_t *i2, uint64_t b2, uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (b2 == 0) { *ob = 0; return OR_OK; }
    if (b0 < 12) return OR_ERR_FORMAT;
    int32_t meta[3];
    memcpy(meta, i0, 12);
    if (meta[0] <= 0 || meta[1] <= 0 || meta[2] < 0) return OR_ERR_FORMAT;
    if ((uint64_t)meta[0] * meta[1] > (1ull << 26)) return OR_ERR_FORMAT;
    gfc_geom_t g;
    int r = gfc_geom(dt, (uint64_t)meta[2], meta[0], meta[1], &g);
    if (r) return r;
    if (b1 < 4ull * g.warps) return OR_ERR_FORMAT;
    if (g.n * es > cap) return OR_ERR_CAP;
    uint64_t pos = 0;
    for (int w = 0; w < g.warps; w++) {
        uint64_t cb = chunk_begin(&g, w), ce = cut_at(&g, w);
        int32_t endabs;
        memcpy(&endabs, i1 + 4 * (uint64_t)w, 4);
        int64_t size = (int64_t)endabs - (int64_t)scratch_start(&g, w);
        if (size < 0 || pos + (uint64_t)size > b2) return OR_ERR_FORMAT;
        uint64_t p = pos, pend = pos + (uint64_t)size;
        uint64_t last = 0, first_last = 0;
        for (uint64_t s = cb; s < ce; s += 32) {
            if (p + 16 > pend) return OR_ERR_FORMAT;
            const uint8_t *hdr = i2 + p;
            p += 16;
            for (int l = 0; l < 32; l++) {
                int nib = (hdr[l / 2] >> (4 * (l & 1))) & 15;
                int code = nib & 7, mb;
                if (dt == OR_DOUBLE) mb = code >= 2 ? code + 1 : code;
                else { mb = code; if (mb > 4) return OR_ERR_FORMAT; }
                if (p + (uint64_t)mb > pend) return OR_ERR_FORMAT;
                uint64_t diff = 0;
                for (int b = mb - 1; b >= 0; b--) diff = (diff << 8) | i2[p + b];
                p += mb;
                if (nib & 8) diff = 0 - diff;
                uint64_t x = last + diff;
                if (dt != OR_DOUBLE) x &= 0xffffffffull;
                if (s + l < g.n) st_u(out, es, s + l, x);
                if (s == cb && l == 31) first_last = x;
            }
            last = first_last;   /* impl_double.cu:146 */
        }
        if (p != pend) return OR_ERR_FORMAT;
        pos = pend;
    }
    *ob = g.n * es;
    return OR_OK;
}
