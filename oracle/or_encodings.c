/*
 * or_encodings.c -- CPU restatement of the reference encodings (AFL, delta, scale, none, RLE,
 * dict/unique, const, patch, floatToInt) and their helpers (stencil, splitter, histogram).
 * TEST INFRASTRUCTURE ONLY (see oracle.h for what pins each part).
 *
 * Compile with -ffp-contract=off: the floating-point expressions below must round exactly like the
 * reference's separately-rounded operations.
 */
#include "or_common.h"

#include <stdio.h>

int or_dtype_size(int dtype) { return es_of(dtype); }

/* ---------------------------------------------------------------- bit lengths ------------- */

/* BITLEN<T>(min, max) -- core/cuda_macros.cuh:168-175 (signed T) */
int or_bitlen(int dtype, int64_t min, int64_t max)
{
    int es = es_of(dtype);
    if (es == 0) return 0;
    if (dtype == OR_FLOAT) return 32;   /* cuda_macros.cuh:185-186 */
    if (dtype == OR_DOUBLE) return 64;  /* cuda_macros.cuh:188-189 */
    if (min < 0) return 8 * es;
    int r = 0;
    while (max >>= 1) r++;
    return r + 1;
}

/* ALT_BITLEN(int) -- core/cuda_macros.cuh:191-205 */
int or_alt_bitlen(int v)
{
    if (v < 0) return 32;
    unsigned r = 0, shift;
    unsigned u = (unsigned)v;
    r = (u > 0xFFFF) << 4; u >>= r;
    shift = (u > 0xFF) << 3; u >>= shift; r |= shift;
    shift = (u > 0xF) << 2; u >>= shift; r |= shift;
    shift = (u > 0x3) << 1; u >>= shift; r |= shift;
    r |= (u >> 1);
    return (int)r + 1;
}

/* ---------------------------------------------------------------- min / max -------------- */

/* CudaArrayStatistics::MinMax (util/statistics/cuda_array_statistics.cu:20-28) with the NaN and
 * signed-zero tie rules spelled out in or_common.h. */
void or_minmax_bits(const uint8_t *p, int dt, uint64_t n, uint64_t *mn, uint64_t *mx)
{
    int es = es_of(dt);
    uint64_t lo = 0, hi = 0;
    int have = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t u = ld_u(p, es, i);
        if (is_nan_bits(u, dt)) continue;
        if (!have) { lo = hi = u; have = 1; continue; }
        if (lt_bits(u, lo, dt)) lo = u;
        else if (!lt_bits(lo, u, dt) && is_fp(dt) && (u >> (8 * es - 1)) && !(lo >> (8 * es - 1)))
            lo = u; /* -0 preferred for min */
        if (lt_bits(hi, u, dt)) hi = u;
        else if (!lt_bits(u, hi, dt) && is_fp(dt) && !(u >> (8 * es - 1)) && (hi >> (8 * es - 1)))
            hi = u; /* +0 preferred for max */
    }
    if (!have && n > 0) lo = hi = ld_u(p, es, 0);
    *mn = lo;
    *mx = hi;
}

/* ---------------------------------------------------------------- stencil ---------------- */

/* Stencil::pack (util/stencil/stencil.cu:14-33, 52-68): [rest = n % 8] then ceil(n/8) bytes, bit
 * i of byte k = element 8k+i; bits past n repeat element n-1 (index clamp at :27). */
uint64_t or_stencil_pack(const int32_t *st, uint64_t n, uint8_t *out)
{
    uint64_t nb = (n + 7) / 8;
    out[0] = (uint8_t)(int8_t)(n % 8);
    for (uint64_t k = 0; k < nb; k++) {
        uint8_t part = 0;
        for (int i = 0; i < 8; i++) {
            uint64_t idx = 8 * k + i;
            if (idx >= n) idx = n - 1;
            if (st[idx] & 1) part |= (uint8_t)(1u << i);
        }
        out[1 + k] = part;
    }
    return nb + 1;
}

/* Stencil::unpack (stencil.cu:35-50, 70-96) */
int64_t or_stencil_unpack(const uint8_t *packed, uint64_t bytes, int32_t *out, uint64_t cap)
{
    if (bytes < 1) return OR_ERR_FORMAT;
    int rest = (int8_t)packed[0];
    int64_t n = (int64_t)(bytes - 1) * 8;
    if (rest) n -= 8 - rest;
    if (n < 0) return OR_ERR_FORMAT;
    if ((uint64_t)n > cap) return OR_ERR_CAP;
    for (int64_t i = 0; i < n; i++) out[i] = (packed[1 + i / 8] >> (i % 8)) & 1;
    return n;
}

/* ---------------------------------------------------------------- splitter --------------- */

void or_split(const uint8_t *in, int es, uint64_t n, const int32_t *st,
              uint8_t *yes, uint64_t *n_yes, uint8_t *no, uint64_t *n_no)
{
    uint64_t a = 0, b = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (st[i]) memcpy(yes + es * a++, in + es * i, es);
        else memcpy(no + es * b++, in + es * i, es);
    }
    *n_yes = a;
    *n_no = b;
}

void or_merge(const uint8_t *yes, const uint8_t *no, int es, const int32_t *st, uint64_t n, uint8_t *out)
{
    uint64_t a = 0, b = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (st[i]) memcpy(out + es * i, yes + es * a++, es);
        else memcpy(out + es * i, no + es * b++, es);
    }
}

/* ---------------------------------------------------------------- sorting / histogram ----- */

void or_radix_sort_u64(uint64_t *keys, uint64_t n)
{
    if (n < 2) return;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *src = keys, *dst = tmp;
    uint64_t *cnt = (uint64_t *)malloc(65536 * sizeof(uint64_t));
    for (int pass = 0; pass < 4; pass++) {
        int sh = 16 * pass;
        memset(cnt, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> sh) & 0xffff]++;
        if (cnt[(src[0] >> sh) & 0xffff] == n) continue;  /* one digit value: the order stands */
        uint64_t s = 0;
        for (int d = 0; d < 65536; d++) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
        for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> sh) & 0xffff]++] = src[i];
        uint64_t *t = src; src = dst; dst = t;
    }
    if (src != keys) memcpy(keys, src, n * sizeof(uint64_t));
    free(cnt);
    free(tmp);
}

typedef struct { uint64_t key; uint64_t cnt; uint64_t order; } bin_t;

static int bin_cmp(const void *a, const void *b)
{
    const bin_t *x = (const bin_t *)a, *y = (const bin_t *)b;
    if (x->cnt != y->cnt) return x->cnt > y->cnt ? -1 : 1;
    return x->order < y->order ? -1 : (x->order > y->order ? 1 : 0);
}

/*
 * Histogram::GetMostFrequent (util/histogram/histogram.cpp:28-35) = ThrustSparseHistogram
 * (thrust_sparse_histogram.cu:19-69: sort, count bins, reduce_by_key) + GetMostFrequentSparse
 * (most_frequent.cu:10-26: stable sort_by_key on counts, greater).  Bins follow same_val();
 * ties are broken by ascending sort order (the stable radix sort keeps the sorted-key order).
 * Slots past the number of distinct values are 0 (the reference leaves them uninitialised).
 */
int or_top_k(const uint8_t *p, int dt, uint64_t n, int k, uint64_t *vals, uint64_t *cnts)
{
    int es = es_of(dt);
    for (int j = 0; j < k; j++) { vals[j] = 0; cnts[j] = 0; }
    if (n == 0) return 0;
    uint64_t *keys = (uint64_t *)malloc(n * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) keys[i] = sort_key(ld_u(p, es, i), dt);
    or_radix_sort_u64(keys, n);
    bin_t *bins = (bin_t *)malloc(n * sizeof(bin_t));
    uint64_t nb = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t u = unsort_key(keys[i], dt);
        if (nb > 0 && same_val(unsort_key(bins[nb - 1].key, dt), u, dt)) { bins[nb - 1].cnt++; continue; }
        bins[nb].key = keys[i]; bins[nb].cnt = 1; bins[nb].order = nb; nb++;
    }
    free(keys);
    qsort(bins, nb, sizeof(bin_t), bin_cmp);
    int m = nb < (uint64_t)k ? (int)nb : k;
    for (int j = 0; j < m; j++) { vals[j] = unsort_key(bins[j].key, dt); cnts[j] = bins[j].cnt; }
    free(bins);
    return m;
}

/* ---------------------------------------------------------------- AFL -------------------- */

/*
 * AflEncoding::Encode<T> (compression/afl/afl_encoding.cu:15-56) with the FL layout of
 * run_afl_compress_gpu<T,1> (afl_gpu.cu:67-73, 124-163): value i occupies bits [i*b, i*b+b) of a
 * little-endian LSB-first bitstream padded to a whole T word.  Metadata [b, rest, 0, 0]; bytes 2-3
 * are uninitialised in the reference and defined as 0 here.
 */
static int afl_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *out,
                      uint64_t cap, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = 0; ob[1] = 0; return OR_OK; }
    uint64_t mnb, mxb;
    or_minmax_bits(in, dt, n, &mnb, &mxb);
    int b = or_bitlen(dt, sext(mnb, es), sext(mxb, es));
    uint64_t W = 8ull * es;
    uint64_t words = (b * n + W - 1) / W;
    uint64_t bytes = words * es;
    if (bytes > cap) return OR_ERR_CAP;
    int8_t rest = (int8_t)(bytes * 8 - n * (uint64_t)b);
    meta[0] = (uint8_t)b; meta[1] = (uint8_t)rest; meta[2] = 0; meta[3] = 0;
    memset(out, 0, bytes);
    uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    /* the bitstream in byte order: whole bytes leave a 128-bit accumulator as soon as they fill */
    unsigned __int128 acc = 0;
    int fill = 0;
    uint8_t *o = out;
    for (uint64_t i = 0; i < n; i++) {
        acc |= (unsigned __int128)(ld_u(in, es, i) & mask) << fill;
        fill += b;
        while (fill >= 8) { *o++ = (uint8_t)acc; acc >>= 8; fill -= 8; }
    }
    if (fill > 0) *o = (uint8_t)acc;
    ob[0] = 4; ob[1] = bytes;
    return OR_OK;
}

/* AflEncoding::Decode<T> / DecodeAfl (afl_encoding.cu:74-113, afl_gpu.cu:165-195) */
static int afl_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *data, uint64_t db,
                      uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (db == 0) { *ob = 0; return OR_OK; }
    if (mb < 2) return OR_ERR_FORMAT;
    int b = (int8_t)meta[0], rest = (int8_t)meta[1];
    if (b <= 0 || b > 8 * es) return OR_ERR_FORMAT;
    int64_t bits = (int64_t)db * 8 - rest;
    if (bits < 0) return OR_ERR_FORMAT;
    uint64_t n = (uint64_t)bits / b;
    if (n * es > cap) return OR_ERR_CAP;
    uint64_t mask = b >= 64 ? ~0ULL : ((1ULL << b) - 1);
    for (uint64_t i = 0; i < n; i++) {
        /* bits [pos, pos + b) of the LSB-first stream: up to 9 bytes from byte pos / 8 */
        uint64_t pos = i * (uint64_t)b, first = pos >> 3;
        unsigned __int128 w = 0;
        int nbytes = (int)((((pos & 7) + (uint64_t)b) + 7) >> 3);
        for (int k = 0; k < nbytes; k++) w |= (unsigned __int128)data[first + k] << (8 * k);
        st_u(out, es, i, (uint64_t)(w >> (pos & 7)) & mask);
    }
    *ob = n * es;
    return OR_OK;
}

/*
 * Bit position of element i of a packed stream, omega = 1 (FL) or 32 (the aligned layout of
 * run_afl_compress_cpu<T,32>, afl_gpu.cu:5-30 and 124-163, addressed as in
 * afl_decompress_base_value_gpu, afl_gpu.cu:197-222): blocks of omega*W elements; element i is row
 * r = (i % omega*W) / omega of lane l = i % omega, and lane l of block B holds its rows LSB first in
 * the words B*omega*b + l + omega*k.  Returns the first bit (in word units: word, bit).
 */
static void afl_locate(int omega, int W, int b, uint64_t i, uint64_t *word, int *bit)
{
    uint64_t per = (uint64_t)omega * W, blk = i / per, in_blk = i % per;
    uint64_t lane = in_blk % omega, row = in_blk / omega;
    *word = blk * omega * (uint64_t)b + lane + (row * b / W) * omega;
    *bit = (int)(row * b % W);
}

uint64_t or_afl_words(int omega, int dtype, int b, uint64_t n)
{
    uint64_t W = 8ull * es_of(dtype);
    if (omega == 1) return (n * b + W - 1) / W;
    return (n + 32 * W - 1) / (32 * W) * 32 * b;
}

/* packs n elements into `words` zeroed words; bits of a value that straddle a word continue at bit
 * 0 of the lane's next word (word + omega) */
int or_afl_pack(int omega, int dtype, int b, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t words)
{
    int es = es_of(dtype), W = 8 * es;
    if (!es || b < 1 || b > W || (omega != 1 && omega != 32)) return OR_ERR_ARG;
    memset(out, 0, words * es);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t w, v = ld_u(in, es, i);
        int bit;
        afl_locate(omega, W, b, i, &w, &bit);
        for (int k = 0; k < b; k++, bit++) {
            if (bit == W) { bit = 0; w += omega; }
            if (w >= words) return OR_ERR_CAP;
            if ((v >> k) & 1) out[w * es + bit / 8] |= (uint8_t)(1u << (bit % 8));
        }
    }
    return OR_OK;
}

/* element idx[t] (or t when idx is NULL) of a packed stream, t < n; bits past `words` read 0 */
int or_afl_values(int omega, int dtype, int b, const uint8_t *comp, uint64_t words, const uint64_t *idx,
                  uint64_t n, uint8_t *out)
{
    int es = es_of(dtype), W = 8 * es;
    if (!es || b < 1 || b > W || (omega != 1 && omega != 32)) return OR_ERR_ARG;
    for (uint64_t t = 0; t < n; t++) {
        uint64_t w, v = 0;
        int bit;
        afl_locate(omega, W, b, idx ? idx[t] : t, &w, &bit);
        for (int k = 0; k < b; k++, bit++) {
            if (bit == W) { bit = 0; w += omega; }
            if (w < words && ((comp[w * es + bit / 8] >> (bit % 8)) & 1)) v |= 1ull << k;
        }
        st_u(out, es, t, v);
    }
    return OR_OK;
}

/* AflEncoding::Encode(SharedCudaPtr<float>) (afl_encoding.cu:116-170): every float is split into
 * its 23-bit mantissa, 8-bit exponent and sign; the mantissa and exponent int32 arrays are AFL
 * packed.  data = mantissa metadata (4) + mantissa words + exponent metadata (4) + exponent words;
 * metadata = size_t mantissa-word bytes, one sign byte (1 all positive, 2 all negative, 0 = the
 * packed stencil of the sign bits follows).  Deviation: "all positive / all negative" is decided
 * on the sign bits; the reference's min >= 0 / max < 0 would drop the sign of -0.0 and of NaNs. */
static int afl_float_encode(const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *out, uint64_t cap,
                            uint64_t ob[3])
{
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    int32_t *mant = (int32_t *)malloc(4 * n), *expo = (int32_t *)malloc(4 * n), *sg = (int32_t *)malloc(4 * n);
    int any1 = 0, all1 = 1;
    for (uint64_t i = 0; i < n; i++) {
        uint32_t u = (uint32_t)ld_u(in, 4, i);
        mant[i] = (int32_t)(u & 0x7fffffu);
        expo[i] = (int32_t)((u >> 23) & 0xffu);
        sg[i] = (int32_t)(u >> 31);
        any1 |= sg[i];
        all1 &= sg[i];
    }
    int sign = !any1 ? 1 : all1 ? 2 : 0;
    uint64_t obm[3], obe[3];
    int r = cap < 8 ? OR_ERR_CAP : afl_encode(OR_INT, (const uint8_t *)mant, n, out, out + 4, cap - 8, obm);
    if (!r) r = afl_encode(OR_INT, (const uint8_t *)expo, n, out + 4 + obm[1], out + 8 + obm[1], cap - 8 - obm[1], obe);
    if (!r) {
        uint64_t msize = obm[1];
        memcpy(meta, &msize, 8);
        meta[8] = (uint8_t)sign;
        ob[0] = 9 + (sign == 0 ? or_stencil_pack(sg, n, meta + 9) : 0);
        ob[1] = 8 + obm[1] + obe[1];
    }
    free(mant);
    free(expo);
    free(sg);
    return r;
}

/* AflEncoding::Decode<float> (afl_encoding.cu:189-254) */
static int afl_float_decode(const uint8_t *meta, uint64_t mb, const uint8_t *data, uint64_t db, uint8_t *out,
                            uint64_t cap, uint64_t *ob)
{
    if (db == 0) { *ob = 0; return OR_OK; }
    if (mb < 9 || db < 8) return OR_ERR_FORMAT;
    uint64_t msize;
    memcpy(&msize, meta, 8);
    int sign = (int8_t)meta[8];
    if (msize > db - 8 || sign < 0 || sign > 2) return OR_ERR_FORMAT;
    uint64_t esize = db - msize - 8;
    uint64_t tcap = 4 * (8 * (msize > esize ? msize : esize) + 8);
    uint8_t *m = (uint8_t *)malloc(tcap), *e = (uint8_t *)malloc(tcap);
    uint64_t obm = 0, obe = 0;
    int r = afl_decode(OR_INT, data, 4, data + 4, msize, m, tcap, &obm);
    if (!r) r = afl_decode(OR_INT, data + 4 + msize, 4, data + 8 + msize, esize, e, tcap, &obe);
    uint64_t n = obm / 4;
    if (!r && obe / 4 < n) r = OR_ERR_FORMAT;
    if (!r && 4 * n > cap) r = OR_ERR_CAP;
    int32_t *sg = NULL;
    if (!r && sign == 0) {
        sg = (int32_t *)malloc(4 * (8 * mb + 8));
        int64_t k = or_stencil_unpack(meta + 9, mb - 9, sg, 8 * mb + 8);
        if (k < (int64_t)n) r = OR_ERR_FORMAT;
    }
    if (!r) {
        for (uint64_t i = 0; i < n; i++) {
            uint32_t s1 = sign == 0 ? (uint32_t)(sg[i] & 1) : (uint32_t)(sign - 1);
            uint32_t u = (s1 << 31) | (((uint32_t)ld_u(e, 4, i) & 0xffu) << 23) | ((uint32_t)ld_u(m, 4, i) & 0x7fffffu);
            st_u(out, 4, i, u);
        }
        *ob = 4 * n;
    }
    free(m);
    free(e);
    free(sg);
    return r;
}

/* ---------------------------------------------------------------- delta / scale / none --- */

/* DeltaEncoding::Encode/Decode (compression/delta/delta_encoding.cu:19-102); float/double go
 * through their int32/int64 bit patterns (delta_encoding.hpp:57-64), so all arithmetic is a
 * wrapping subtraction / addition of raw element bits. */
static int delta_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *out, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    memcpy(meta, in, es);
    for (uint64_t i = 0; i + 1 < n; i++) st_u(out, es, i, ld_u(in, es, i + 1) - ld_u(in, es, i));
    ob[0] = es; ob[1] = (n - 1) * es;
    return OR_OK;
}

static int delta_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *d, uint64_t db,
                        uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (mb == 0) { *ob = 0; return OR_OK; }
    if (mb < (uint64_t)es) return OR_ERR_FORMAT;
    uint64_t n = db / es + 1;
    if (n * es > cap) return OR_ERR_CAP;
    uint64_t acc = ld_u(meta, es, 0);
    st_u(out, es, 0, acc);
    for (uint64_t i = 1; i < n; i++) { acc += ld_u(d, es, i - 1); st_u(out, es, i, acc); }
    *ob = n * es;
    return OR_OK;
}

/* ScaleEncoding::Encode/Decode (compression/scale/scale_encoding.cu:21-108; float/double as
 * int32/int64, scale_encoding.hpp:48-55).  The overflow test at :49-50 is evaluated with the
 * wrap-around an x86 build gives for int/long. */
static int scale_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *out, uint64_t ob[3])
{
    int es = es_of(dt);
    int idt = dt == OR_FLOAT ? OR_INT : (dt == OR_DOUBLE ? OR_TIME : dt);
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    uint64_t mnb, mxb;
    or_minmax_bits(in, idt, n, &mnb, &mxb);
    int64_t mn = sext(mnb, es), mx = sext(mxb, es);
    if (mn < 0) {
        if (es <= 2) {
            int64_t tmax = es == 1 ? 127 : 32767;
            if ((tmax - mx) < (mn < 0 ? -mn : mn)) mn = 0;
        } else {
            uint64_t W = 8ull * es;
            uint64_t m = W == 64 ? ~0ULL : ((1ULL << W) - 1);
            uint64_t tmax = m >> 1;
            int64_t diff = sext((tmax - (uint64_t)mx) & m, es);
            int64_t absmn = sext((0 - (uint64_t)mn) & m, es);
            if (diff < absmn) mn = 0;
        }
    }
    st_u(meta, es, 0, (uint64_t)mn);
    for (uint64_t i = 0; i < n; i++) st_u(out, es, i, ld_u(in, es, i) - (uint64_t)mn);
    ob[0] = es; ob[1] = n * es;
    return OR_OK;
}

static int scale_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *d, uint64_t db,
                        uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (db == 0) { *ob = 0; return OR_OK; }
    if (mb < (uint64_t)es) return OR_ERR_FORMAT;
    uint64_t n = db / es;
    if (n * es > cap) return OR_ERR_CAP;
    uint64_t mn = ld_u(meta, es, 0);
    for (uint64_t i = 0; i < n; i++) st_u(out, es, i, ld_u(d, es, i) + mn);
    *ob = n * es;
    return OR_OK;
}

/* NoneEncoding (compression/none/none_encoding.cu:13-49): metadata = size_t byte count. */
static int none_encode(const uint8_t *in, uint64_t in_bytes, uint8_t *meta, uint8_t *out, uint64_t ob[3])
{
    memcpy(meta, &in_bytes, 8);
    memcpy(out, in, in_bytes);
    ob[0] = 8; ob[1] = in_bytes;
    return OR_OK;
}

/* ---------------------------------------------------------------- RLE -------------------- */

/* RleEncoding::Encode (compression/rle/rle_encode.cu:18-62): reduce_by_key over equal neighbours
 * (same_val), meta = int32 run count, out1 = int32 lengths, out2 = T values. */
static int rle_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint8_t *o2, uint64_t ob[3])
{
    int es = es_of(dt);
    int32_t runs = 0;
    uint64_t i = 0;
    while (i < n) {
        uint64_t u = ld_u(in, es, i), j = i + 1;
        while (j < n && same_val(u, ld_u(in, es, j), dt)) j++;
        int32_t len = (int32_t)(j - i);
        memcpy(o1 + 4 * (uint64_t)runs, &len, 4);
        st_u(o2, es, runs, u);
        runs++;
        i = j;
    }
    memcpy(meta, &runs, 4);
    ob[0] = 4; ob[1] = 4 * (uint64_t)runs; ob[2] = (uint64_t)es * runs;
    return OR_OK;
}

/* RleEncoding::Decode (compression/rle/rle_decode.cu:19-73) */
static int rle_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *l, uint64_t lb,
                      const uint8_t *v, uint64_t vb, uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (lb == 0) { *ob = 0; return OR_OK; }
    if (mb < 4) return OR_ERR_FORMAT;
    int32_t runs;
    memcpy(&runs, meta, 4);
    if (runs < 0 || (uint64_t)runs * 4 > lb || (uint64_t)runs * es > vb) return OR_ERR_FORMAT;
    uint64_t pos = 0;
    for (int32_t r = 0; r < runs; r++) {
        int32_t len;
        memcpy(&len, l + 4 * (uint64_t)r, 4);
        if (len < 0) return OR_ERR_FORMAT;
        if ((pos + (uint64_t)len) * es > cap) return OR_ERR_CAP;
        uint64_t u = ld_u(v, es, r);
        for (int32_t k = 0; k < len; k++) st_u(out, es, pos++, u);
    }
    *ob = pos * es;
    return OR_OK;
}

/* ---------------------------------------------------------------- unique coder ----------- */

/*
 * UniqueEncoding::CompressUnique (compression/unique/unique_encoding.cu:48-76, 88-131): header
 * size_t uniqueCnt, size_t m, T table[uniqueCnt], then uint32 words holding 32/bits codes each
 * (code of value i at bits [bits*(i%per), ...) of word i/per).  A value's code is the OR of every
 * table index it matches.  Code slots past m (an out-of-bounds read in the reference) are 0.
 */
static uint64_t unique_compress(int dt, const uint8_t *data, uint64_t m, const uint64_t *table, int tcnt, uint8_t *out)
{
    int es = es_of(dt);
    if (m == 0) return 0;
    int bits = or_alt_bitlen(tcnt - 1);
    int per = 32 / bits;
    uint64_t words = (m + per - 1) / per;
    uint64_t hdr = 16 + (uint64_t)tcnt * es;
    uint64_t sz[2] = {(uint64_t)tcnt, m};
    memcpy(out, sz, 16);
    for (int j = 0; j < tcnt; j++) st_u(out + 16, es, j, table[j]);
    for (uint64_t w = 0; w < words; w++) {
        uint32_t word = 0;
        for (int i = 0; i < per; i++) {
            uint64_t idx = w * per + i;
            if (idx >= m) break;
            uint64_t u = ld_u(data, es, idx);
            for (int j = 0; j < tcnt; j++)
                if (same_val(u, table[j], dt)) word |= (uint32_t)j << (bits * i);
        }
        memcpy(out + hdr + 4 * w, &word, 4);
    }
    return hdr + 4 * words;
}

/* UniqueEncoding::DecompressUnique (unique_encoding.cu:183-259) */
static int64_t unique_decompress(int dt, const uint8_t *in, uint64_t bytes, uint8_t *out, uint64_t cap)
{
    int es = es_of(dt);
    if (bytes == 0) return 0;
    if (bytes < 16) return OR_ERR_FORMAT;
    uint64_t sz[2];
    memcpy(sz, in, 16);
    uint64_t tcnt = sz[0], m = sz[1];
    if (tcnt == 0 || tcnt > (1u << 30)) return OR_ERR_FORMAT;
    int bits = or_alt_bitlen((int)tcnt - 1);
    int per = 32 / bits;
    uint64_t hdr = 16 + tcnt * es;
    uint64_t words = (m + per - 1) / per;
    if (hdr + 4 * words > bytes) return OR_ERR_FORMAT;
    if (m * es > cap) return OR_ERR_CAP;
    for (uint64_t i = 0; i < m; i++) {
        uint32_t word;
        memcpy(&word, in + hdr + 4 * (i / per), 4);
        uint32_t code = (word >> (bits * (i % per))) & (bits == 32 ? 0xffffffffu : ((1u << bits) - 1));
        if (code >= tcnt) return OR_ERR_FORMAT;
        memcpy(out + es * i, in + 16 + es * (uint64_t)code, es);
    }
    return (int64_t)(m * es);
}

/* ---------------------------------------------------------------- dict ------------------- */

/* DictEncoding::Encode (compression/dict/dict_encoding.cu:15-95), _freqCnt = 4 */
static int dict_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint8_t *o2, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = ob[2] = 0; return OR_OK; }
    uint64_t top[4], cnt[4];
    or_top_k(in, dt, n, 4, top, cnt);
    int32_t *st = (int32_t *)malloc(n * sizeof(int32_t));
    for (uint64_t i = 0; i < n; i++) {
        uint64_t u = ld_u(in, es, i);
        int hit = 0;
        for (int j = 0; j < 4; j++) hit |= same_val(u, top[j], dt);
        st[i] = hit;
    }
    uint8_t *yes = (uint8_t *)malloc(n * es), *no = o2;
    uint64_t ny, nn;
    or_split(in, es, n, st, yes, &ny, no, &nn);
    ob[0] = or_stencil_pack(st, n, meta);
    ob[1] = unique_compress(dt, yes, ny, top, 4, o1);
    ob[2] = nn * es;
    free(st);
    free(yes);
    return OR_OK;
}

/* DictEncoding::Decode (dict_encoding.cu:103-130) */
static int dict_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *i1, uint64_t b1,
                       const uint8_t *i2, uint64_t b2, uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (b1 == 0 && b2 == 0) { *ob = 0; return OR_OK; }
    uint64_t maxn = mb * 8;
    int32_t *st = (int32_t *)malloc((maxn + 1) * sizeof(int32_t));
    int64_t n = or_stencil_unpack(meta, mb, st, maxn);
    if (n < 0) { free(st); return (int)n; }
    if ((uint64_t)n * es > cap) { free(st); return OR_ERR_CAP; }
    uint8_t *yes = (uint8_t *)malloc((uint64_t)n * es + 8);
    int64_t yb = unique_decompress(dt, i1, b1, yes, (uint64_t)n * es);
    if (yb < 0) { free(st); free(yes); return (int)yb; }
    uint64_t nyes = 0;
    for (int64_t i = 0; i < n; i++) nyes += st[i] != 0;
    if ((uint64_t)yb < nyes * es || b2 < ((uint64_t)n - nyes) * es) { free(st); free(yes); return OR_ERR_FORMAT; }
    or_merge(yes, i2, es, st, (uint64_t)n, out);
    *ob = (uint64_t)n * es;
    free(st);
    free(yes);
    return OR_OK;
}

/* Standalone UniqueEncoding (unique_encoding.cu:35-46, 133-181, 261-304).  The table holds every
 * distinct bit pattern in sort order (NaN payloads and signed zeros kept apart so the coding is
 * lossless; the reference's float `==` maps NaN to code 0). */
static int unique_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    uint64_t *keys = (uint64_t *)malloc(n * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) keys[i] = sort_key(ld_u(in, es, i), dt);
    or_radix_sort_u64(keys, n);
    uint64_t u = 0;
    for (uint64_t i = 0; i < n; i++)
        if (i == 0 || keys[i] != keys[u - 1]) keys[u++] = keys[i];
    int bits = or_alt_bitlen((int)u - 1);
    int per = 32 / bits;
    uint64_t words = (n + per - 1) / per;
    uint64_t sz[2] = {u, n};
    memcpy(meta, sz, 16);
    for (uint64_t j = 0; j < u; j++) st_u(meta + 16, es, j, unsort_key(keys[j], dt));
    for (uint64_t w = 0; w < words; w++) {
        uint32_t word = 0;
        for (int i = 0; i < per && w * per + i < n; i++) {
            uint64_t k = sort_key(ld_u(in, es, w * per + i), dt);
            uint64_t lo = 0, hi = u;
            while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (keys[mid] < k) lo = mid + 1; else hi = mid; }
            word |= (uint32_t)lo << (bits * i);
        }
        memcpy(o1 + 4 * w, &word, 4);
    }
    free(keys);
    ob[0] = 16 + u * es; ob[1] = 4 * words;
    return OR_OK;
}

static int unique_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *d, uint64_t db,
                         uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (db == 0) { *ob = 0; return OR_OK; }
    if (mb < 16) return OR_ERR_FORMAT;
    uint64_t sz[2];
    memcpy(sz, meta, 16);
    uint64_t u = sz[0], n = sz[1];
    if (u == 0 || 16 + u * es > mb) return OR_ERR_FORMAT;
    int bits = or_alt_bitlen((int)u - 1);
    int per = 32 / bits;
    if ((n + per - 1) / per * 4 > db) return OR_ERR_FORMAT;
    if (n * es > cap) return OR_ERR_CAP;
    uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t word;
        memcpy(&word, d + 4 * (i / per), 4);
        uint32_t code = (word >> (bits * (i % per))) & mask;
        if (code >= u) return OR_ERR_FORMAT;
        memcpy(out + es * i, meta + 16 + es * (uint64_t)code, es);
    }
    *ob = n * es;
    return OR_OK;
}

/* ---------------------------------------------------------------- const ------------------ */

/* ConstEncoding::Encode/Decode (compression/const/const_encoding.cu:19-131): meta = T c ||
 * packed stencil of (x is not c), data = the non-c values in order. */
static int const_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    uint64_t top, cnt;
    or_top_k(in, dt, n, 1, &top, &cnt);
    int32_t *st = (int32_t *)malloc(n * sizeof(int32_t));
    for (uint64_t i = 0; i < n; i++) st[i] = !same_val(ld_u(in, es, i), top, dt);
    uint64_t a = 0;
    for (uint64_t i = 0; i < n; i++)
        if (st[i]) memcpy(o1 + es * a++, in + es * i, es);
    st_u(meta, es, 0, top);
    ob[0] = es + or_stencil_pack(st, n, meta + es);
    ob[1] = a * es;
    free(st);
    return OR_OK;
}

static int const_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *d, uint64_t db,
                        uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (mb == 0) { *ob = 0; return OR_OK; }
    if (mb < (uint64_t)es + 1) return OR_ERR_FORMAT;
    uint64_t maxn = (mb - es) * 8;
    int32_t *st = (int32_t *)malloc((maxn + 1) * sizeof(int32_t));
    int64_t n = or_stencil_unpack(meta + es, mb - es, st, maxn);
    if (n < 0) { free(st); return (int)n; }
    if ((uint64_t)n * es > cap) { free(st); return OR_ERR_CAP; }
    uint64_t c = ld_u(meta, es, 0), a = 0;
    for (int64_t i = 0; i < n; i++) {
        if (st[i]) {
            if ((a + 1) * es > db) { free(st); return OR_ERR_FORMAT; }
            memcpy(out + es * i, d + es * a++, es);
        } else st_u(out, es, i, c);
    }
    *ob = (uint64_t)n * es;
    free(st);
    return OR_OK;
}

/* ---------------------------------------------------------------- patch ------------------ */

/* static_cast<T>(double) as the reference's x86 host build evaluates it */
static uint64_t cast_double_to_T(double d, int dt)
{
    switch (dt) {
    case OR_FLOAT: return f32_bits((float)d);
    case OR_DOUBLE: return f64_bits(d);
    case OR_TIME: return (uint64_t)cvtt_i64(d);
    default: return (uint64_t)(int64_t)cvtt_i32(d);
    }
}

/* T value (raw bits) -> double, as the LowerPatchEncoding(double min, double max) constructor
 * receives it (patch_encoding_factory.hpp:46-55) */
static double T_to_double(uint64_t u, int dt)
{
    switch (dt) {
    case OR_FLOAT: return (double)bits_f32((uint32_t)u);
    case OR_DOUBLE: return bits_f64(u);
    default: return (double)sext(u, es_of(dt));
    }
}

/* threshold of LowerPatchEncoding::GetOperator<T> (lower_patch_encoding.cu:22-31), factor 0.1 */
static uint64_t lower_patch_threshold(uint64_t mnb, uint64_t mxb, int dt)
{
    double dmin = T_to_double(mnb, dt), dmax = T_to_double(mxb, dt);
    uint64_t dist_bits = cast_double_to_T(dmax - dmin, dt);   /* T dist = _max - _min; */
    double ddist = T_to_double(dist_bits, dt);
    if (dt != OR_FLOAT && dt != OR_DOUBLE) ddist = (double)sext(dist_bits, es_of(dt));
    double prod = 0.1 * ddist;
    double t = dmax - prod;
    return cast_double_to_T(t, dt);
}

/* bounds of OutsidePatchEncoding::GetOperator<T> (outside_patch_encoding.cu:22-31), factor 0.1:
 * T dist = _max - _min; low = static_cast<T>(_min + 0.1 * dist), high = static_cast<T>(_max - 0.1 * dist) */
static void outside_patch_bounds(uint64_t mnb, uint64_t mxb, int dt, uint64_t *lo, uint64_t *hi)
{
    double dmin = T_to_double(mnb, dt), dmax = T_to_double(mxb, dt);
    uint64_t dist_bits = cast_double_to_T(dmax - dmin, dt);
    double ddist = T_to_double(dist_bits, dt);
    if (dt != OR_FLOAT && dt != OR_DOUBLE) ddist = (double)sext(dist_bits, es_of(dt));
    double prod = 0.1 * ddist;
    *lo = cast_double_to_T(dmin + prod, dt);
    *hi = cast_double_to_T(dmax - prod, dt);
}

/* PatchEncodingFactory<T>::Get(data) (patch_encoding_factory.hpp:40-57) + LowerPatchEncoding
 * (lower_patch_encoding.cu:33-94): stencil x < t, meta = packed stencil, out1 = x < t values,
 * out2 = the rest, both in order.  With `outside`, OutsidePatchEncoding::Encode
 * (outside_patch_encoding.cu:33-60): stencil = OutsideOperator (stencil_operators.hpp:14-25),
 * true unless x > high or x < low (so NaN is true), same three outputs.  Empty input: three empty
 * buffers for both variants. */
static int patch_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint8_t *o2, uint64_t ob[3],
                        int outside)
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = ob[2] = 0; return OR_OK; }
    uint64_t mnb, mxb;
    or_minmax_bits(in, dt, n, &mnb, &mxb);
    uint64_t t = lower_patch_threshold(mnb, mxb, dt), lo = 0, hi = 0;
    if (outside) outside_patch_bounds(mnb, mxb, dt, &lo, &hi);
    int32_t *st = (int32_t *)malloc(n * sizeof(int32_t));
    for (uint64_t i = 0; i < n; i++) {
        uint64_t x = ld_u(in, es, i);
        st[i] = outside ? !(lt_bits(hi, x, dt) || lt_bits(x, lo, dt)) : lt_bits(x, t, dt);
    }
    uint64_t ny, nn;
    or_split(in, es, n, st, o1, &ny, o2, &nn);
    ob[0] = or_stencil_pack(st, n, meta);
    ob[1] = ny * es; ob[2] = nn * es;
    free(st);
    return OR_OK;
}

/* Lower/OutsidePatchEncoding::Decode (lower_patch_encoding.cu:69-94) */
static int patch_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *i1, uint64_t b1,
                        const uint8_t *i2, uint64_t b2, uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (b1 == 0 && b2 == 0) { *ob = 0; return OR_OK; }
    uint64_t maxn = mb * 8;
    int32_t *st = (int32_t *)malloc((maxn + 1) * sizeof(int32_t));
    int64_t n = or_stencil_unpack(meta, mb, st, maxn);
    if (n < 0) { free(st); return (int)n; }
    if ((uint64_t)n * es > cap) { free(st); return OR_ERR_CAP; }
    uint64_t ny = 0;
    for (int64_t i = 0; i < n; i++) ny += st[i] != 0;
    if (ny * es > b1 || ((uint64_t)n - ny) * es > b2) { free(st); return OR_ERR_FORMAT; }
    or_merge(i1, i2, es, st, (uint64_t)n, out);
    *ob = (uint64_t)n * es;
    free(st);
    return OR_OK;
}

/* ---------------------------------------------------------------- floatToInt ------------- */

static const double kPow10[10] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9};

/* IntegerToFloatingPointOperator<int,T> (util/transform/transform_operators.hpp:121-131):
 * (T)x / pow(10, p), the quotient rounded to T on return. */
static uint64_t f2i_decode_one(int32_t k, int p, int dt)
{
    double q;
    switch (dt) {
    case OR_FLOAT: q = (double)(float)k / kPow10[p]; return f32_bits((float)q);
    case OR_DOUBLE: q = (double)k / kPow10[p]; return f64_bits(q);
    case OR_TIME: q = (double)(int64_t)k / kPow10[p]; return (uint64_t)cvtt_i64(q);
    default: {
        int es = es_of(dt);
        int64_t t = sext((uint64_t)(int64_t)k, es); /* (T)x truncates to the element width */
        q = (double)t / kPow10[p];
        return (uint64_t)(int64_t)cvtt_i32(q);
    }
    }
}

/*
 * FloatEncoding::Encode/Decode (compression/float/float_encoding.cu:17-88) with
 * FloatingPointToIntegerOperator (transform_operators.hpp:109-119): p = Precision(data); if p < 10
 * and min*10^p > INT_MIN and max*10^p < INT_MAX the data becomes lrint(x * 10^p) as int32, else
 * p = 10 and the raw bytes are kept.  Deviation, to stay lossless: when any element would not
 * decode to its exact input bits the encoder takes the p = 10 branch (the reference's stream would
 * have lost those bits).
 */
static int f2i_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *meta, uint8_t *o1, uint64_t ob[3])
{
    int es = es_of(dt);
    if (n == 0) { ob[0] = ob[1] = 0; return OR_OK; }
    int p = 0;
    for (uint64_t i = 0; i < n; i++) {
        int q = or_float_precision(ld_f32(in, dt, i));
        if (q > p) p = q;
    }
    int transform = 0;
    if (p < 10) {
        uint64_t mnb, mxb;
        or_minmax_bits(in, dt, n, &mnb, &mxb);
        int scale = (int)kPow10[p];
        int ok;
        if (dt == OR_FLOAT) {
            float a = bits_f32((uint32_t)mnb) * (float)scale, b = bits_f32((uint32_t)mxb) * (float)scale;
            ok = a > (float)INT32_MIN && b < (float)INT32_MAX;
        } else if (dt == OR_DOUBLE) {
            double a = bits_f64(mnb) * (double)scale, b = bits_f64(mxb) * (double)scale;
            ok = a > (double)INT32_MIN && b < (double)INT32_MAX;
        } else {
            int64_t a = sext(mnb, es), b = sext(mxb, es);
            ok = a * scale > INT32_MIN && b * scale < INT32_MAX;
        }
        if (ok) transform = 1; else p = 10;
    }
    if (transform) {
        uint64_t wmask = es == 8 ? ~0ull : ((1ull << (8 * es)) - 1);
        for (uint64_t i = 0; i < n; i++) {
            double x = ld_num(in, dt, i);
            int32_t k = (int32_t)(int64_t)llrint(x * kPow10[p]);
            if (((f2i_decode_one(k, p, dt) ^ ld_u(in, es, i)) & wmask) != 0) { transform = 0; p = 10; break; }
            memcpy(o1 + 4 * i, &k, 4);
        }
    }
    memcpy(meta, &p, 4);
    ob[0] = 4;
    if (transform) ob[1] = 4 * n;
    else {
        uint64_t bytes = (n * es) / 4 * 4;   /* CastSharedCudaPtr<T,int> keeps whole ints */
        memcpy(o1, in, bytes);
        ob[1] = bytes;
    }
    return OR_OK;
}

static int f2i_decode(int dt, const uint8_t *meta, uint64_t mb, const uint8_t *d, uint64_t db,
                      uint8_t *out, uint64_t cap, uint64_t *ob)
{
    int es = es_of(dt);
    if (db == 0) { *ob = 0; return OR_OK; }
    if (mb < 4) return OR_ERR_FORMAT;
    int32_t p;
    memcpy(&p, meta, 4);
    if (p < 10) {
        if (p < 0) return OR_ERR_FORMAT;
        uint64_t n = db / 4;
        if (n * es > cap) return OR_ERR_CAP;
        for (uint64_t i = 0; i < n; i++) {
            int32_t k;
            memcpy(&k, d + 4 * i, 4);
            st_u(out, es, i, f2i_decode_one(k, p, dt));
        }
        *ob = n * es;
    } else {
        uint64_t n = db / es;
        if (n * es > cap) return OR_ERR_CAP;
        memcpy(out, d, n * es);
        *ob = n * es;
    }
    return OR_OK;
}

/* ---------------------------------------------------------------- dispatch --------------- */

int or_gfc_encode(int dt, const uint8_t *in, uint64_t n, uint8_t *o0, uint8_t *o1, uint8_t *o2, uint64_t ob[3]);
int or_gfc_decode(int dt, const uint8_t *i0, uint64_t b0, const uint8_t *i1, uint64_t b1,
                  const uint8_t *i2, uint64_t b2, uint8_t *out, uint64_t cap, uint64_t *ob);

static uint64_t worst_case(int enc, int dt, uint64_t in_bytes)
{
    int es = es_of(dt);
    uint64_t n = in_bytes / (es ? es : 1);
    switch (enc) {
    case OR_GFC: return in_bytes + n / 2 + 4096 + 4 * ((n + 32767) / 32768 + 1) * 32;
    case OR_UNIQUE: return 16 + in_bytes + 4 * n + 64;
    case OR_RLE: return 4 * n + in_bytes + 64;
    default: return 2 * in_bytes + n / 8 + 64;
    }
}

int or_encode(int enc, int dt, const uint8_t *in, uint64_t in_bytes,
              uint8_t *o0, uint8_t *o1, uint8_t *o2, uint64_t cap,
              uint64_t ob[3], int *n_out)
{
    int es = es_of(dt);
    if (!es) return OR_ERR_TYPE;
    if (cap < worst_case(enc, dt, in_bytes) && enc != OR_NONE) return OR_ERR_CAP;
    uint64_t n = in_bytes / es;
    ob[0] = ob[1] = ob[2] = 0;
    switch (enc) {
    case OR_AFL:
        *n_out = 2;
        if (dt == OR_FLOAT) return afl_float_encode(in, n, o0, o1, cap, ob);
        if (is_fp(dt)) return OR_ERR_UNSUPPORTED;  /* EncodeDouble returns no buffers at all */
        return afl_encode(dt, in, n, o0, o1, cap, ob);
    case OR_DELTA: *n_out = 2; return delta_encode(dt, in, n, o0, o1, ob);
    case OR_SCALE: *n_out = 2; return scale_encode(dt, in, n, o0, o1, ob);
    case OR_NONE:
        if (cap < in_bytes || cap < 8) return OR_ERR_CAP;
        *n_out = 2; return none_encode(in, in_bytes, o0, o1, ob);
    case OR_RLE: *n_out = 3; return rle_encode(dt, in, n, o0, o1, o2, ob);
    case OR_DICT: *n_out = 3; return dict_encode(dt, in, n, o0, o1, o2, ob);
    case OR_UNIQUE: *n_out = 2; return unique_encode(dt, in, n, o0, o1, ob);
    case OR_CONST: *n_out = 2; return const_encode(dt, in, n, o0, o1, ob);
    case OR_PATCH: *n_out = 3; return patch_encode(dt, in, n, o0, o1, o2, ob, 0);
    case OR_PATCH_OUTSIDE: *n_out = 3; return patch_encode(dt, in, n, o0, o1, o2, ob, 1);
    case OR_FLOAT2INT: *n_out = 2; return f2i_encode(dt, in, n, o0, o1, ob);
    case OR_GFC:
        if (!is_fp(dt)) {
            int r = afl_encode(dt, in, n, o0, o1, cap, ob);
            *n_out = 3; ob[2] = 0;
            return r;
        }
        *n_out = 3; return or_gfc_encode(dt, in, n, o0, o1, o2, ob);
    default: return OR_ERR_ARG;
    }
}

int or_decode(int enc, int dt, const uint8_t *i0, uint64_t b0, const uint8_t *i1, uint64_t b1,
              const uint8_t *i2, uint64_t b2, uint8_t *out, uint64_t cap, uint64_t *ob)
{
    if (!es_of(dt)) return OR_ERR_TYPE;
    *ob = 0;
    switch (enc) {
    case OR_AFL:
        if (dt == OR_FLOAT) return afl_float_decode(i0, b0, i1, b1, out, cap, ob);
        if (is_fp(dt)) return OR_ERR_UNSUPPORTED;
        return afl_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_DELTA: return delta_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_SCALE: return scale_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_NONE:
        if (b1 > cap) return OR_ERR_CAP;
        memcpy(out, i1, b1); *ob = b1; return OR_OK;
    case OR_RLE: return rle_decode(dt, i0, b0, i1, b1, i2, b2, out, cap, ob);
    case OR_DICT: return dict_decode(dt, i0, b0, i1, b1, i2, b2, out, cap, ob);
    case OR_UNIQUE: return unique_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_CONST: return const_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_PATCH: case OR_PATCH_OUTSIDE: return patch_decode(dt, i0, b0, i1, b1, i2, b2, out, cap, ob);
    case OR_FLOAT2INT: return f2i_decode(dt, i0, b0, i1, b1, out, cap, ob);
    case OR_GFC:
        if (!is_fp(dt)) return afl_decode(dt, i0, b0, i1, b1, out, cap, ob);
        return or_gfc_decode(dt, i0, b0, i1, b1, i2, b2, out, cap, ob);
    default: return OR_ERR_ARG;
    }
}
