/*
 * or_common.h -- element access and conversion helpers shared by the oracle's C files.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#ifndef GTSC_OR_COMMON_H_
#define GTSC_OR_COMMON_H_

#include "oracle.h"
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int es_of(int dt)
{
    switch (dt) {
    case OR_CHAR: return 1;
    case OR_SHORT: return 2;
    case OR_INT: case OR_FLOAT: return 4;
    case OR_TIME: case OR_DOUBLE: return 8;
    default: return 0;
    }
}

static inline int is_fp(int dt) { return dt == OR_FLOAT || dt == OR_DOUBLE; }

/* raw bits of element i, zero-extended */
static inline uint64_t ld_u(const uint8_t *p, int es, uint64_t i)
{
    switch (es) {
    case 1: return p[i];
    case 2: { uint16_t v; memcpy(&v, p + 2 * i, 2); return v; }
    case 4: { uint32_t v; memcpy(&v, p + 4 * i, 4); return v; }
    default: { uint64_t v; memcpy(&v, p + 8 * i, 8); return v; }
    }
}

static inline void st_u(uint8_t *p, int es, uint64_t i, uint64_t v)
{
    switch (es) {
    case 1: p[i] = (uint8_t)v; break;
    case 2: { uint16_t w = (uint16_t)v; memcpy(p + 2 * i, &w, 2); } break;
    case 4: { uint32_t w = (uint32_t)v; memcpy(p + 4 * i, &w, 4); } break;
    default: memcpy(p + 8 * i, &v, 8); break;
    }
}

/* raw bits sign-extended from the element width (the "integer view" of any element) */
static inline int64_t sext(uint64_t v, int es)
{
    switch (es) {
    case 1: return (int8_t)v;
    case 2: return (int16_t)v;
    case 4: return (int32_t)v;
    default: return (int64_t)v;
    }
}

static inline int64_t ld_s(const uint8_t *p, int es, uint64_t i) { return sext(ld_u(p, es, i), es); }

static inline float bits_f32(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline double bits_f64(uint64_t u) { double f; memcpy(&f, &u, 8); return f; }
static inline uint32_t f32_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline uint64_t f64_bits(double f) { uint64_t u; memcpy(&u, &f, 8); return u; }

/* numeric value of element i as double (exact for every type except int64 beyond 2^53) */
static inline double ld_num(const uint8_t *p, int dt, uint64_t i)
{
    switch (dt) {
    case OR_FLOAT: return (double)bits_f32((uint32_t)ld_u(p, 4, i));
    case OR_DOUBLE: return bits_f64(ld_u(p, 8, i));
    case OR_TIME: return (double)ld_s(p, 8, i);
    default: return (double)ld_s(p, es_of(dt), i);
    }
}

/* element i converted to float the way the reference's (float)x casts round (directly from T) */
static inline float ld_f32(const uint8_t *p, int dt, uint64_t i)
{
    switch (dt) {
    case OR_FLOAT: return bits_f32((uint32_t)ld_u(p, 4, i));
    case OR_DOUBLE: return (float)bits_f64(ld_u(p, 8, i));
    case OR_TIME: return (float)ld_s(p, 8, i);
    default: return (float)ld_s(p, es_of(dt), i);
    }
}

static inline int is_nan_bits(uint64_t u, int dt)
{
    if (dt == OR_FLOAT) return ((u >> 23) & 0xff) == 0xff && (u & 0x7fffff) != 0;
    if (dt == OR_DOUBLE) return ((u >> 52) & 0x7ff) == 0x7ff && (u & 0xfffffffffffffULL) != 0;
    return 0;
}

/* T-native "<" of two elements given as raw bits */
static inline int lt_bits(uint64_t a, uint64_t b, int dt)
{
    switch (dt) {
    case OR_FLOAT: return bits_f32((uint32_t)a) < bits_f32((uint32_t)b);
    case OR_DOUBLE: return bits_f64(a) < bits_f64(b);
    default: { int es = es_of(dt); return sext(a, es) < sext(b, es); }
    }
}

/*
 * Value identity used by RLE runs, histogram bins and dictionary matching.  For integer types it
 * is the reference's `==`.  For floating types it is `==` AND equal bits: identical to the
 * reference except that -0.0 and +0.0 are kept apart (the reference merges them and so loses the
 * sign of zero).  NaN never matches, as in the reference.
 */
static inline int same_val(uint64_t a, uint64_t b, int dt)
{
    if (a != b) return 0;
    return !is_nan_bits(a, dt);
}

/* monotone unsigned sort key: signed order for integers, radix "twiddle" order for floats */
static inline uint64_t sort_key(uint64_t u, int dt)
{
    switch (dt) {
    case OR_FLOAT: { uint32_t v = (uint32_t)u; return (v & 0x80000000u) ? (uint32_t)~v : (v | 0x80000000u); }
    case OR_DOUBLE: return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
    default: { int es = es_of(dt); return u ^ (1ULL << (8 * es - 1)); }
    }
}
static inline uint64_t unsort_key(uint64_t k, int dt)
{
    switch (dt) {
    case OR_FLOAT: { uint32_t v = (uint32_t)k; return (v & 0x80000000u) ? (v & 0x7fffffffu) : (uint32_t)~v; }
    case OR_DOUBLE: return (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    default: { int es = es_of(dt); return k ^ (1ULL << (8 * es - 1)); }
    }
}

/* x86-64 cvttsd2si semantics (what the reference's host-side double->integer casts compile to):
 * truncation toward zero, and the "integer indefinite" value for NaN / out-of-range inputs. */
static inline int32_t cvtt_i32(double d)
{
    if (!(d > -2147483649.0 && d < 2147483648.0)) return INT32_MIN;
    return (int32_t)d;
}
static inline int64_t cvtt_i64(double d)
{
    if (!(d >= -9223372036854775808.0 && d < 9223372036854775808.0)) return INT64_MIN;
    return (int64_t)d;
}

/* Stable min/max of a typed array in T-native order.  Floating NaNs are skipped unless every
 * element is NaN (then both are element 0); among equal values (+-0) min prefers -0, max +0.
 * Returns raw bits. */
void or_minmax_bits(const uint8_t *p, int dt, uint64_t n, uint64_t *mn, uint64_t *mx);

/* histogram top-k: values (raw bits) ordered by count desc, then sort_key asc; unused slots 0 */
int or_top_k(const uint8_t *p, int dt, uint64_t n, int k, uint64_t *vals, uint64_t *cnts);

/* stable split / merge by a 0/1 stencil (util/splitter/splitter.cu:66-184) */
void or_split(const uint8_t *in, int es, uint64_t n, const int32_t *st,
              uint8_t *yes, uint64_t *n_yes, uint8_t *no, uint64_t *n_no);
void or_merge(const uint8_t *yes, const uint8_t *no, int es, const int32_t *st, uint64_t n, uint8_t *out);

void or_radix_sort_u64(uint64_t *keys, uint64_t n);

#endif
