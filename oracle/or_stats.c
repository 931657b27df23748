/*
 * or_stats.c -- CPU restatement of CudaArrayStatistics (util/statistics/cuda_array_statistics.cu).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include "or_common.h"

/* _getFloatPrecision (cuda_array_statistics.cu:37-44): smallest e = 10^k (k <= 10) with
 * round(x*e)/e == x in float arithmetic, reported as (int)(logf(e)/logf(10)). */
int or_float_precision(float x)
{
    long e = 1;
    const long maxp = 10000000000L;
    while (1) {
        float fe = (float)e;
        float prod = x * fe;
        float rq = roundf(prod) / fe;
        if (!(rq != x && e < maxp)) break;
        e *= 10;
    }
    volatile float a = logf((float)e), b = logf(10.0f);
    volatile float q = a / b;
    return (int)q;
}

/* device float/double -> int conversion (cvt.rzi.s32): truncate, saturate, NaN -> 0 */
static inline int32_t dev_f2i(double d)
{
    if (d != d) return 0;
    if (d >= 2147483647.0) return INT32_MAX;
    if (d <= -2147483648.0) return INT32_MIN;
    return (int32_t)d;
}

/* `int value = data[idx]` of _rlMetricKernel, then `value == data[idx+i]` in T arithmetic.  The
 * kernel runs on the device, so the conversion is the device's cvt.rzi.s32: measured on the B200,
 * a float NaN converts to 0 and a double NaN to INT_MIN (tests/test_encodings_gpu.py pins both). */
static inline int32_t rl_to_int(uint64_t u, int dt)
{
    switch (dt) {
    case OR_FLOAT: return dev_f2i((double)bits_f32((uint32_t)u));
    case OR_DOUBLE: { double d = bits_f64(u); return d != d ? INT32_MIN : dev_f2i(d); }
    case OR_TIME: return (int32_t)(uint32_t)u;
    default: return (int32_t)sext(u, es_of(dt));
    }
}
static inline int rl_eq(int32_t v, uint64_t u, int dt)
{
    switch (dt) {
    case OR_FLOAT: return (float)v == bits_f32((uint32_t)u);
    case OR_DOUBLE: return (double)v == bits_f64(u);
    case OR_TIME: return (int64_t)v == (int64_t)u;
    default: return (int64_t)v == sext(u, es_of(dt));
    }
}

/* RlMetric<T,N> (cuda_array_statistics.cu:97-132) */
float or_rl_metric(int dt, const uint8_t *in, uint64_t in_bytes, int N)
{
    int es = es_of(dt);
    uint64_t n = in_bytes / es;
    if ((uint64_t)N >= n) return 1.0f;
    uint64_t m = n - N;
    int64_t sum = 0;
    for (uint64_t idx = 0; idx < m; idx++) {
        int32_t v = rl_to_int(ld_u(in, es, idx), dt);
        int num = 1, out = 1, last = 1;
        for (int i = 1; i < N; i++) {
            out = rl_eq(v, ld_u(in, es, idx + i), dt);
            num += out & last;
            last = out;
        }
        sum += num;
    }
    return (float)((double)(int32_t)sum / (double)m);
}

/* Mean<T> (cuda_array_statistics.cu:134-139): sum in T arithmetic (wrapping for integers), then
 * sum / (double)n converted back to T.  Floating sums are order dependent in the reference
 * (thrust::reduce); here they are summed left to right. */
static double mean_of(const uint8_t *in, int dt, uint64_t n)
{
    int es = es_of(dt);
    if (dt == OR_FLOAT) {
        float s = 0;
        for (uint64_t i = 0; i < n; i++) s += bits_f32((uint32_t)ld_u(in, 4, i));
        return (double)(float)(s / (double)n);
    }
    if (dt == OR_DOUBLE) {
        double s = 0;
        for (uint64_t i = 0; i < n; i++) s += bits_f64(ld_u(in, 8, i));
        return s / (double)n;
    }
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) s += ld_u(in, es, i);
    int64_t ss = sext(s & (es == 8 ? ~0ull : ((1ull << (8 * es)) - 1)), es);
    double q = (double)ss / (double)n;
    if (dt == OR_TIME) return (double)cvtt_i64(q);
    return (double)sext((uint64_t)(int64_t)cvtt_i32(q), es);
}

/* GenerateStatistics -> getStatistics<T> (cuda_array_statistics.cu:141-179) */
int or_stats(int dt, const uint8_t *in, uint64_t in_bytes, or_stats_t *s)
{
    int es = es_of(dt);
    if (!es) return OR_ERR_TYPE;
    memset(s, 0, sizeof(*s));
    uint64_t n = in_bytes / es;
    s->size = n;
    if (n == 0) return OR_OK;
    uint64_t mnb, mxb;
    or_minmax_bits(in, dt, n, &mnb, &mxb);
    s->min = dt == OR_FLOAT ? (double)bits_f32((uint32_t)mnb) : dt == OR_DOUBLE ? bits_f64(mnb) : (double)sext(mnb, es);
    s->max = dt == OR_FLOAT ? (double)bits_f32((uint32_t)mxb) : dt == OR_DOUBLE ? bits_f64(mxb) : (double)sext(mxb, es);
    s->min_bit_cnt = 64;   /* BITLEN<double> specialisation, cuda_macros.cuh:188-189 */
    int p = 0;
    for (uint64_t i = 0; i < n; i++) {
        int q = or_float_precision(ld_f32(in, dt, i));
        if (q > p) p = q;
    }
    s->precision = p;
    int sorted = 1;
    for (uint64_t i = 0; i + 1 < n; i++)
        if (lt_bits(ld_u(in, es, i + 1), ld_u(in, es, i), dt)) { sorted = 0; break; }
    s->sorted = sorted;
    s->rl_metric = or_rl_metric(dt, in, in_bytes, 2);
    s->mean = mean_of(in, dt, n);
    return OR_OK;
}
