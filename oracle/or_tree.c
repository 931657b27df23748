/*
 * or_tree.c -- CPU restatement of the compression tree (serialize / deserialize / size prediction)
 * and of the plain exhaustive planner.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include "or_common.h"

#include <stdio.h>

#define MAX_DEPTH 64

/* GetNumberOfResults of each encoding (the *_encoding.hpp headers under compression/) */
static int nres(int enc)
{
    switch (enc) {
    case OR_DELTA: case OR_AFL: case OR_SCALE: case OR_UNIQUE: case OR_FLOAT2INT: case OR_CONST: return 1;
    case OR_RLE: case OR_DICT: case OR_PATCH: case OR_PATCH_OUTSIDE: case OR_GFC: return 2;
    case OR_NONE: return 0;
    default: return -1;
    }
}

/* GetReturnTypes: rle {int, T} (rle_encoding.hpp:35), floatToInt {int} (float_encoding.hpp:31),
 * everything else {T, T} */
static int ret_type(int enc, int dt, int j)
{
    if (enc == OR_RLE && j == 0) return OR_INT;
    if (enc == OR_FLOAT2INT) return OR_INT;
    return dt;
}

/* room for any encoding's outputs: RLE of 1-byte values writes 4 bytes of run length per value */
static uint64_t enc_cap(uint64_t in_bytes) { return 5 * in_bytes + 8192; }

/* ---------------------------------------------------------------- path -> tree ------------ */

static int from_path_rec(const int16_t *encs, int n, int *id, int dt, int16_t *nodes, int cap, int *cnt, int depth)
{
    if (*id >= n || depth > MAX_DEPTH) return OR_ERR_FORMAT;
    int enc = encs[*id];
    int r = nres(enc);
    if (r < 0 || es_of(dt) == 0) return OR_ERR_ARG;
    if (*cnt >= cap) return OR_ERR_CAP;
    nodes[2 * *cnt] = (int16_t)enc;
    nodes[2 * *cnt + 1] = (int16_t)dt;
    (*cnt)++;
    for (int j = 0; j < r; j++) {
        (*id)++;
        int e = from_path_rec(encs, n, id, ret_type(enc, dt, j), nodes, cap, cnt, depth + 1);
        if (e) return e;
    }
    return OR_OK;
}

int or_tree_from_path(const int16_t *encs, int n_encs, int dtype, int16_t *nodes, int cap)
{
    int id = 0, cnt = 0;
    int e = from_path_rec(encs, n_encs, &id, dtype, nodes, cap, &cnt, 0);
    if (e) return e;
    if (id != n_encs - 1) return OR_ERR_FORMAT;
    return cnt;
}

/* ---------------------------------------------------------------- compress --------------- */

typedef struct {
    const int16_t *nodes;
    int n, pos;
} cursor_t;

/* CompressionNode::Compress (tree/compression_node.cpp:103-138) + PrepareMetadata (:84-101) */
static int compress_rec(cursor_t *c, const uint8_t *in, uint64_t in_bytes, uint8_t *out, uint64_t cap,
                        uint64_t *w, int depth)
{
    if (c->pos >= c->n || depth > MAX_DEPTH) return OR_ERR_FORMAT;
    int enc = c->nodes[2 * c->pos], dt = c->nodes[2 * c->pos + 1];
    c->pos++;
    int r = nres(enc);
    if (r < 0 || es_of(dt) == 0) return OR_ERR_ARG;
    uint64_t ec = enc_cap(in_bytes);
    uint8_t *o[3];
    for (int j = 0; j < 3; j++) o[j] = (uint8_t *)malloc(ec);
    uint64_t ob[3];
    int n_out = 0;
    int e = or_encode(enc, dt, in, in_bytes, o[0], o[1], o[2], ec, ob, &n_out);
    if (!e) {
        if (*w + 8 + ob[0] > cap) e = OR_ERR_CAP;
    }
    if (!e) {
        /* both patch variants serialise as EncodingType::patch */
        int16_t hdr16[2] = {(int16_t)(enc == OR_PATCH_OUTSIDE ? OR_PATCH : enc), (int16_t)dt};
        int32_t ml = (int32_t)ob[0];
        memcpy(out + *w, hdr16, 4);
        memcpy(out + *w + 4, &ml, 4);
        memcpy(out + *w + 8, o[0], ob[0]);
        *w += 8 + ob[0];
        if (enc == OR_NONE) {
            if (*w + ob[1] > cap) e = OR_ERR_CAP;
            else { memcpy(out + *w, o[1], ob[1]); *w += ob[1]; }
        } else {
            for (int j = 0; j < r && !e; j++) e = compress_rec(c, o[j + 1], ob[j + 1], out, cap, w, depth + 1);
        }
    }
    for (int j = 0; j < 3; j++) free(o[j]);
    return e;
}

int or_tree_compress(const int16_t *nodes, int n_nodes, const uint8_t *in, uint64_t in_bytes,
                     uint8_t *out, uint64_t cap, uint64_t *out_bytes)
{
    cursor_t c = {nodes, n_nodes, 0};
    uint64_t w = 0;
    int e = compress_rec(&c, in, in_bytes, out, cap, &w, 0);
    if (e) return e;
    if (c.pos != n_nodes) return OR_ERR_FORMAT;
    *out_bytes = w;
    return OR_OK;
}

/* ---------------------------------------------------------------- decompress ------------- */

/* upper bound of a node's decoded bytes, read from its inputs (never trusted beyond the blob) */
static uint64_t decode_bound(int enc, int dt, const uint8_t *i0, uint64_t b0, uint64_t b1, const uint8_t *i1)
{
    int es = es_of(dt);
    switch (enc) {
    case OR_NONE: case OR_SCALE: return b1;
    case OR_DELTA: return b1 + es;
    case OR_AFL: return b1 * 8 * es;
    case OR_GFC:
        if (!is_fp(dt)) return b1 * 8 * es;
        if (b0 >= 12) { int32_t m[3]; memcpy(m, i0, 12); if (m[2] >= 0) return (uint64_t)m[2] * es; }
        return 0;
    case OR_RLE: {
        uint64_t s = 0;
        for (uint64_t k = 0; k + 4 <= b1; k += 4) { int32_t l; memcpy(&l, i1 + k, 4); if (l > 0) s += (uint64_t)l; }
        return s * es;
    }
    case OR_DICT: case OR_PATCH: return b0 * 8 * es;
    case OR_CONST: return b0 * 8 * es;
    case OR_UNIQUE: if (b0 >= 16) { uint64_t sz[2]; memcpy(sz, i0, 16); return sz[1] * es; } return 0;
    case OR_FLOAT2INT: return (b1 / 4 + 1) * 8;
    default: return 0;
    }
}

/* DecompressNodes + CompressionNode::Decompress (tree/compression_tree.cpp:105-146,
 * compression_node.cpp:140-161) */
static int decompress_rec(const uint8_t *blob, uint64_t bytes, uint64_t *off, uint8_t **res, uint64_t *res_bytes,
                          int *dt_out, uint64_t limit, int depth)
{
    if (depth > MAX_DEPTH) return OR_ERR_FORMAT;
    if (*off + 8 > bytes) return OR_ERR_FORMAT;
    int16_t h[2];
    int32_t ml;
    memcpy(h, blob + *off, 4);
    memcpy(&ml, blob + *off + 4, 4);
    *off += 8;
    int enc = h[0], dt = h[1];
    int r = nres(enc);
    if (r < 0 || es_of(dt) == 0 || ml < 0 || *off + (uint64_t)ml > bytes) return OR_ERR_FORMAT;
    const uint8_t *meta = blob + *off;
    *off += (uint64_t)ml;
    *dt_out = dt;
    if (enc == OR_NONE) {
        if (ml < 8) return OR_ERR_FORMAT;
        uint64_t ds;
        memcpy(&ds, meta, 8);
        if (ds > bytes - *off) return OR_ERR_FORMAT;
        *res = (uint8_t *)malloc(ds ? ds : 1);
        memcpy(*res, blob + *off, ds);
        *res_bytes = ds;
        *off += ds;
        return OR_OK;
    }
    uint8_t *ch[2] = {0, 0};
    uint64_t cb[2] = {0, 0};
    int e = OR_OK;
    for (int j = 0; j < r && !e; j++) {
        int cdt;
        e = decompress_rec(blob, bytes, off, &ch[j], &cb[j], &cdt, limit, depth + 1);
    }
    if (!e) {
        uint64_t bound = decode_bound(enc, dt, meta, (uint64_t)ml, cb[0], ch[0]);
        if (bound > limit) e = OR_ERR_CAP;
        else {
            *res = (uint8_t *)malloc(bound + 8);
            e = or_decode(enc, dt, meta, (uint64_t)ml, ch[0], cb[0], ch[1], cb[1], *res, bound + 8, res_bytes);
            if (e) { free(*res); *res = 0; }
        }
    }
    free(ch[0]);
    free(ch[1]);
    return e;
}

int or_tree_decompress(const uint8_t *blob, uint64_t blob_bytes, uint8_t *out, uint64_t cap,
                       uint64_t *out_bytes, int *dtype)
{
    uint64_t off = 0, rb = 0;
    uint8_t *res = 0;
    int dt = 0;
    int e = decompress_rec(blob, blob_bytes, &off, &res, &rb, &dt, 64 * (blob_bytes + cap) + (1u << 20), 0);
    if (e) return e;
    if (off != blob_bytes) { free(res); return OR_ERR_FORMAT; }
    if (rb > cap) { free(res); return OR_ERR_CAP; }
    memcpy(out, res, rb);
    free(res);
    *out_bytes = rb;
    *dtype = dt;
    return OR_OK;
}

/* ---------------------------------------------------------------- size prediction -------- */

/* Encoding::GetMetadataSize of each encoding for `bytes` of input of type dt */
static int meta_size(int enc, int dt, const uint8_t *in, uint64_t bytes, uint64_t *ms)
{
    int es = es_of(dt);
    uint64_t elems = bytes / es;
    switch (enc) {
    case OR_NONE: *ms = 8; return OR_OK;                                   /* none_encoding.hpp:36-39 */
    case OR_DELTA: case OR_SCALE: *ms = bytes ? (uint64_t)es : 0; return OR_OK;
    case OR_RLE: case OR_FLOAT2INT: *ms = bytes ? 4 : 0; return OR_OK;
    case OR_AFL:                                                          /* afl_encoding.cu:281-293 */
        if (!bytes) { *ms = 0; return OR_OK; }
        if (dt == OR_INT) { *ms = 4; return OR_OK; }
        if (dt == OR_FLOAT) { *ms = 9; return OR_OK; }
        return OR_ERR_UNSUPPORTED;
    case OR_DICT: *ms = (elems + 7) / 8 + 1; return OR_OK;               /* dict_encoding.hpp:44-48 */
    case OR_PATCH: case OR_PATCH_OUTSIDE: *ms = bytes ? (elems + 7) / 8 + 1 : 0; return OR_OK;
    case OR_CONST: *ms = bytes ? (elems + 7) / 8 + es + 1 : 0; return OR_OK;
    case OR_GFC: *ms = 12; return OR_OK;
    case OR_UNIQUE: {
        if (!bytes) { *ms = 0; return OR_OK; }
        uint64_t ob[3]; int no;
        uint64_t cap = enc_cap(bytes) + 16 * elems;
        uint8_t *a = (uint8_t *)malloc(cap), *b = (uint8_t *)malloc(cap), *c = (uint8_t *)malloc(cap);
        int e = or_encode(OR_UNIQUE, dt, in, bytes, a, b, c, cap, ob, &no);
        free(a); free(b); free(c);
        if (e) return e;
        *ms = ob[0];
        return OR_OK;
    }
    default: return OR_ERR_ARG;
    }
}

static int predict_rec(cursor_t *c, int type, const uint8_t *in, uint64_t bytes, uint64_t *size, int depth)
{
    if (c->pos >= c->n || depth > MAX_DEPTH) return OR_ERR_FORMAT;
    int enc = c->nodes[2 * c->pos];
    c->pos++;
    int r = nres(enc);
    if (r < 0) return OR_ERR_ARG;
    uint64_t ms;
    int e = meta_size(enc, type, in, bytes, &ms);
    if (e) return e;
    *size += ms + 8;
    if (enc == OR_NONE) { *size += bytes; return OR_OK; }  /* NoneEncoding::GetCompressedSize */
    uint64_t ec = enc_cap(bytes);
    uint8_t *o[3];
    for (int j = 0; j < 3; j++) o[j] = (uint8_t *)malloc(ec);
    uint64_t ob[3];
    int n_out;
    e = or_encode(enc, type, in, bytes, o[0], o[1], o[2], ec, ob, &n_out);
    for (int j = 0; j < r && !e; j++) e = predict_rec(c, ret_type(enc, type, j), o[j + 1], ob[j + 1], size, depth + 1);
    for (int j = 0; j < 3; j++) free(o[j]);
    return e;
}

int or_tree_predict_size(const int16_t *nodes, int n_nodes, const uint8_t *in, uint64_t in_bytes, uint64_t *size)
{
    if (n_nodes <= 0) return OR_ERR_ARG;
    cursor_t c = {nodes, n_nodes, 0};
    *size = 0;
    int e = predict_rec(&c, nodes[1], in, in_bytes, size, 0);
    if (e) return e;
    return c.pos == n_nodes ? OR_OK : OR_ERR_FORMAT;
}

/* ---------------------------------------------------------------- exhaustive planner ----- */

#define MAX_LEVEL 3   /* optimizer/path_generator.cpp:15 */

/* PathGenerator::GetContinuations (optimizer/path_generator.cpp:93-146).  `whole` = the input is a
 * whole number of elements of its type; when it is not (a dictionary's code stream re-read as 8-byte
 * values), every encoding but none would drop its last bytes (CastSharedCudaPtr), so only none is
 * offered: a deliberate departure that keeps every planned tree lossless. */
static int continuations(int et, int dt, const or_stats_t *s, int level, int whole, int *out)
{
    int k = 0;
    if (level != 0 && (et == OR_NONE || s->size == 0)) return 0;
    out[k++] = OR_NONE;
    if (et == OR_AFL || et == OR_GFC || !whole) return k;
    if (level < MAX_LEVEL) {
        if (et != OR_DELTA) out[k++] = OR_DELTA;
        if (et != OR_SCALE && s->min != 0) out[k++] = OR_SCALE;
        if (et != OR_FLOAT2INT && dt == OR_FLOAT) out[k++] = OR_FLOAT2INT;
        if (et != OR_PATCH && et != OR_DICT) out[k++] = OR_PATCH;
        if (et != OR_DICT && et != OR_PATCH) out[k++] = OR_DICT;
        if (s->sorted || s->rl_metric >= 1.5f) {
            if (et != OR_CONST) out[k++] = OR_CONST;
            if (et != OR_RLE) out[k++] = OR_RLE;
        }
    }
    out[k++] = is_fp(dt) ? OR_GFC : OR_AFL;
    return k;
}

typedef struct {
    uint64_t size;
    int n;
    int16_t *nodes;
} cand_t;

static void cand_set_leaf(cand_t *c, int enc, int dt, uint64_t size)
{
    /* a parent-only candidate, Fix()ed: `none` children carry the parent's data type
     * (compression_node.cpp:211-219) */
    int r = nres(enc);
    c->n = 1 + r;
    c->nodes = (int16_t *)realloc(c->nodes, sizeof(int16_t) * 2 * c->n);
    c->nodes[0] = (int16_t)enc; c->nodes[1] = (int16_t)dt;
    for (int j = 0; j < r; j++) { c->nodes[2 + 2 * j] = OR_NONE; c->nodes[3 + 2 * j] = (int16_t)dt; }
    c->size = size;
}

/*
 * FullStatisticsUpdate (compression_optimizer.cpp:88-140) reduced to its best candidate: sizes of
 * crossed subtrees add up, so the minimum-size candidate of a call is made of the minimum-size
 * candidates of its children, and the first minimum in the reference's enumeration order
 * (continuations in order, cross products left-major) is the concatenation of the children's
 * first minima.  Returns 0 when the reference would return an empty list.
 */
static int fsu(const uint8_t *data, uint64_t bytes, int et, int dt, int level, cand_t *best)
{
    or_stats_t st;
    or_stats(dt, data, bytes, &st);
    int cont[16];
    int nc = continuations(et, dt, &st, level, bytes % es_of(dt) == 0, cont);
    if (nc == 0) return 0;
    best->size = UINT64_MAX;
    uint64_t ec = enc_cap(bytes);
    for (int ci = 0; ci < nc; ci++) {
        int c = cont[ci];
        uint8_t *o[3];
        for (int j = 0; j < 3; j++) o[j] = (uint8_t *)malloc(ec);
        uint64_t ob[3] = {0, 0, 0};
        int n_out = 0;
        cand_t cand = {0, 0, 0};
        int e = or_encode(c, dt, data, bytes, o[0], o[1], o[2], ec, ob, &n_out);
        if (e) {
            fprintf(stderr, "oracle fsu: encode %d dt %d failed %d\n", c, dt, e);
            for (int j = 0; j < 3; j++) free(o[j]);
            continue;
        }
        uint64_t psize = 8;
        for (int j = 0; j < n_out; j++) psize += ob[j];
        int r = nres(c);
        cand_t ch[2] = {{0, 0, 0}, {0, 0, 0}};
        int ok = r > 0;
        for (int j = 0; j < r; j++) ok = fsu(o[j + 1], ob[j + 1], c, ret_type(c, dt, j), level + 1, &ch[j]) && ok;
        if (r == 0 || !ok) cand_set_leaf(&cand, c, dt, psize);
        else {
            cand.n = 1;
            for (int j = 0; j < r; j++) cand.n += ch[j].n;
            cand.nodes = (int16_t *)malloc(sizeof(int16_t) * 2 * cand.n);
            cand.nodes[0] = (int16_t)c; cand.nodes[1] = (int16_t)dt;
            int k = 1;
            cand.size = ob[0] + 8;
            for (int j = 0; j < r; j++) {
                memcpy(cand.nodes + 2 * k, ch[j].nodes, sizeof(int16_t) * 2 * ch[j].n);
                k += ch[j].n;
                cand.size += ch[j].size;
            }
        }
        free(ch[0].nodes);
        free(ch[1].nodes);
        if (cand.size < best->size) {
            free(best->nodes);
            *best = cand;
        } else free(cand.nodes);
        for (int j = 0; j < 3; j++) free(o[j]);
    }
    return 1;
}

uint64_t or_sample_bytes(int dtype, uint64_t in_bytes)
{
    int es = es_of(dtype);
    if (!es) return 0;
    uint64_t n = in_bytes / es;
    return n <= 10000 ? in_bytes : 10000ull * es;
}

int or_plan_exhaustive(int dtype, const uint8_t *in, uint64_t in_bytes,
                       int16_t *nodes_out, int cap, int *n_nodes, uint64_t *best_size)
{
    if (!es_of(dtype)) return OR_ERR_TYPE;
    cand_t best = {0, 0, 0};
    fsu(in, in_bytes, OR_NONE, dtype, 0, &best);
    /* std::max_element over GetCompressionRatio (compression_optimizer.cpp:174-177): ratios saturate
     * at 1.0, so a candidate only beats the leading `none` tree when it is strictly smaller than
     * the input. */
    if (!(best.size < in_bytes)) cand_set_leaf(&best, OR_NONE, dtype, in_bytes + 16);
    if (best.n > cap) { free(best.nodes); return OR_ERR_CAP; }
    memcpy(nodes_out, best.nodes, sizeof(int16_t) * 2 * best.n);
    *n_nodes = best.n;
    *best_size = best.size;
    free(best.nodes);
    return OR_OK;
}

/* PathGenerator::GeneratePaths (optimizer/path_generator.cpp:20-68): 6 x 5 paths */
static int gen_path(int idx, int16_t *p)
{
    static const int16_t first[6][2] = {{-1, -1}, {OR_FLOAT2INT, -1}, {OR_DELTA, -1}, {OR_SCALE, -1},
                                        {OR_DELTA, OR_FLOAT2INT}, {OR_SCALE, OR_FLOAT2INT}};
    static const int16_t second[5][5] = {
        {OR_DICT, OR_AFL, OR_NONE, OR_AFL, OR_NONE},
        {OR_CONST, OR_AFL, OR_NONE, -1, -1},
        {OR_RLE, OR_AFL, OR_NONE, OR_AFL, OR_NONE},
        {OR_AFL, OR_NONE, -1, -1, -1},
        {OR_PATCH, OR_AFL, OR_NONE, OR_AFL, OR_NONE}};
    int k = 0, a = idx / 5, b = idx % 5;
    for (int j = 0; j < 2; j++) if (first[a][j] >= 0) p[k++] = first[a][j];
    for (int j = 0; j < 5; j++) if (second[b][j] >= 0) p[k++] = second[b][j];
    return k;
}

int or_optimize_tree(int dtype, const uint8_t *in, uint64_t in_bytes,
                     int16_t *nodes_out, int cap, int *n_nodes, uint64_t *best_size)
{
    if (!es_of(dtype)) return OR_ERR_TYPE;
    uint64_t min_size = in_bytes;
    int16_t best[64];
    int best_n = 1;
    best[0] = OR_NONE; best[1] = (int16_t)dtype;
    for (int i = 0; i < 30; i++) {
        int16_t path[8], nodes[64];
        int pl = gen_path(i, path);
        int nn = or_tree_from_path(path, pl, dtype, nodes, 32);
        if (nn < 0) return nn;
        uint64_t sz;
        if (or_tree_predict_size(nodes, nn, in, in_bytes, &sz)) continue;  /* reference would throw */
        if (sz < min_size) { min_size = sz; memcpy(best, nodes, sizeof(int16_t) * 2 * nn); best_n = nn; }
    }
    if (best_n > cap) return OR_ERR_CAP;
    memcpy(nodes_out, best, sizeof(int16_t) * 2 * best_n);
    *n_nodes = best_n;
    *best_size = min_size;
    return OR_OK;
}
