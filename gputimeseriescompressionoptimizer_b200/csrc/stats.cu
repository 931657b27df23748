// stats.cu -- column statistics in one pass (CudaArrayStatistics::GenerateStatistics,
// util/statistics/cuda_array_statistics.cu:141-179) and the floatToInt transform
// (FloatEncoding, compression/float/float_encoding.cu:17-88).
//
// The reference launches MinMax, Precision, Sorted, RlMetric<T,2> and Mean as five separate
// passes, each followed by a device-to-host read (Precision alone ran at ~0.5 GB/s on its GPU).
// Here one kernel reads every element once and folds all five statistics; the host reads one
// small accumulator.
//
// Precision: _getFloatPrecision (cuda_array_statistics.cu:37-44) multiplies by e = 10^k until
// round(x*e)/e == x (float arithmetic, k <= 10) and reports (int)(logf(e)/logf(10)).  The kernel
// records the number of steps k per element (IEEE-rounded __fmul_rn / roundf / __fdiv_rn, the
// operations the reference's loop performs) and the maximum k is mapped through a table that
// k_log_table computes once with CUDA's own logf.
#include "kernels.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int ST_THREADS = 256;

__device__ __forceinline__ int precision_steps(float x)
{
    long long e = 1;
    int k = 0;
    while (true) {
        const float fe = (float)e;
        const float q = __fdiv_rn(roundf(__fmul_rn(x, fe)), fe);
        if (!(q != x && e < 10000000000ll)) break;
        e *= 10;
        ++k;
    }
    return k;
}

template <int ES>
__device__ __forceinline__ float as_float(uint64_t u, Order o)
{
    if (o == ORD_F32) return __uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __double2float_rn(__longlong_as_double((long long)u));
    if (ES == 8) return __ll2float_rn((long long)u);
    return __int2float_rn((int)sext(u, ES));
}

// `int value = data[idx]` of _rlMetricKernel: device conversion (truncate, saturate, NaN -> 0)
template <int ES>
__device__ __forceinline__ int rl_int(uint64_t u, Order o)
{
    if (o == ORD_F32) return __float2int_rz(__uint_as_float((uint32_t)u));
    if (o == ORD_F64) return __double2int_rz(__longlong_as_double((long long)u));
    // integer types: sign-extended from the element width, 64-bit values keep their low 32 bits
    return ES == 8 ? (int)(uint32_t)u : (int)sext(u, ES);
}
template <int ES>
__device__ __forceinline__ bool rl_eq(int v, uint64_t u, Order o)
{
    if (o == ORD_F32) return __int2float_rn(v) == __uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __int2double_rn(v) == __longlong_as_double((long long)u);
    return (long long)v == sext(u, ES);
}

template <int ES>
__global__ void __launch_bounds__(ST_THREADS)
k_stats(const uint8_t *__restrict__ in, uint64_t n, Order o, StatsAcc *acc, double *fsum_partial)
{
    uint64_t kmin = ~0ull, kmax = 0;
    int kprec = 0;
    bool unsorted = false;
    unsigned long long rl = 0, isum = 0;
    double fsum = 0.0;  // float columns accumulate in float below, double columns in double
    float fsum32 = 0.0f;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    {
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const uint64_t u = ld_elem<ES>(in, i);
            if (!is_nan_bits(u, o)) {
                const uint64_t k = order_key(u, ES, o);
                kmin = k < kmin ? k : kmin;
                kmax = k > kmax ? k : kmax;
            }
            const int p = precision_steps(as_float<ES>(u, o));
            kprec = p > kprec ? p : kprec;
            if (i + 1 < n) {
                const uint64_t nx = ld_elem<ES>(in, i + 1);
                if (lt_native(nx, u, ES, o)) unsorted = true;
                if (i + 2 < n) rl += 1ull + (rl_eq<ES>(rl_int<ES>(u, o), nx, o) ? 1ull : 0ull);
            }
            if (o == ORD_F32) fsum32 += __uint_as_float((uint32_t)u);
            else if (o == ORD_F64) fsum += __longlong_as_double((long long)u);
            else isum += u;
        }
    }
    if (o == ORD_F32) fsum = fsum32;
    // block reduction
    __shared__ unsigned long long s_min[ST_THREADS / 32], s_max[ST_THREADS / 32], s_rl[ST_THREADS / 32],
        s_isum[ST_THREADS / 32];
    __shared__ int s_prec[ST_THREADS / 32], s_uns[ST_THREADS / 32];
    __shared__ double s_f[ST_THREADS];
    s_f[threadIdx.x] = fsum;
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, kmin, off);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, kmax, off);
        kmin = a < kmin ? a : kmin;
        kmax = b > kmax ? b : kmax;
        rl += __shfl_xor_sync(0xffffffffu, rl, off);
        isum += __shfl_xor_sync(0xffffffffu, isum, off);
        const int p = __shfl_xor_sync(0xffffffffu, kprec, off);
        kprec = p > kprec ? p : kprec;
        unsorted = __any_sync(0xffffffffu, unsorted);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_min[warp] = kmin; s_max[warp] = kmax; s_rl[warp] = rl; s_isum[warp] = isum;
        s_prec[warp] = kprec; s_uns[warp] = unsorted;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < ST_THREADS / 32; w++) {
            kmin = s_min[w] < kmin ? s_min[w] : kmin;
            kmax = s_max[w] > kmax ? s_max[w] : kmax;
            rl += s_rl[w];
            isum += s_isum[w];
            kprec = s_prec[w] > kprec ? s_prec[w] : kprec;
            unsorted |= s_uns[w] != 0;
        }
        if (kmin != ~0ull) atomicMax(&acc->mm.nkmin, (unsigned long long)~kmin);
        if (kmax != 0) atomicMax(&acc->mm.kmax, (unsigned long long)kmax);
        atomicAdd(&acc->rl_sum, rl);
        atomicAdd(&acc->int_sum, isum);
        atomicMax(&acc->prec_steps, (unsigned int)kprec);
        if (unsorted) atomicExch(&acc->unsorted, 1u);
        // floating sums: in thread order inside the block, blocks combined in order on the host
        if (o == ORD_F32) {
            float s = 0.0f;
            for (int t = 0; t < ST_THREADS; t++) s += (float)s_f[t];
            fsum_partial[blockIdx.x] = s;
        } else {
            double s = 0.0;
            for (int t = 0; t < ST_THREADS; t++) s += s_f[t];
            fsum_partial[blockIdx.x] = s;
        }
    }
}

__global__ void k_log_table(int *table)
{
    const int k = threadIdx.x;
    if (k > 10) return;
    long long e = 1;
    for (int i = 0; i < k; i++) e *= 10;
    const float q = logf((float)e) / logf(10.0f);
    table[k] = (int)q;
}

// ------------------------------------------------------------------------------ floatToInt
__device__ __constant__ double kPow10[10] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9};

template <int ES>
__device__ __forceinline__ double as_double(uint64_t u, Order o)
{
    if (o == ORD_F32) return (double)__uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __longlong_as_double((long long)u);
    if (ES == 8) return __ll2double_rn((long long)u);
    return (double)sext(u, ES);
}

// IntegerToFloatingPointOperator (util/transform/transform_operators.hpp:121-131)
template <int ES>
__device__ __forceinline__ uint64_t f2i_decode_one(int k, int p, Order o)
{
    if (o == ORD_F32) {
        const double q = __ddiv_rn((double)__int2float_rn(k), kPow10[p]);
        return __float_as_uint(__double2float_rn(q));
    }
    if (o == ORD_F64) return (uint64_t)__double_as_longlong(__ddiv_rn((double)k, kPow10[p]));
    if (ES == 8) return (uint64_t)__double2ll_rz(__ddiv_rn((double)k, kPow10[p]));
    const long long t = sext((uint64_t)(long long)k, ES);
    return (uint64_t)(long long)__double2int_rz(__ddiv_rn((double)t, kPow10[p]));
}

template <int ES>
__global__ void __launch_bounds__(ST_THREADS)
k_f2i_encode(const uint8_t *__restrict__ in, uint64_t n, Order o, int p, int32_t *__restrict__ out,
             unsigned int *__restrict__ lossy)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t wmask = ES == 8 ? ~0ull : ((1ull << (8 * ES)) - 1);
    bool bad = false;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t u = ld_elem<ES>(in, i);
        const int k = (int)(long long)__double2ll_rn(__dmul_rn(as_double<ES>(u, o), kPow10[p]));
        out[i] = k;
        if (((f2i_decode_one<ES>(k, p, o) ^ u) & wmask) != 0) bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(lossy, 1u);
}

template <int ES>
__global__ void __launch_bounds__(ST_THREADS)
k_f2i_decode(const uint8_t *__restrict__ in, uint64_t n, Order o, int p, uint8_t *__restrict__ out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int k = (int)ld_elem<4>(in, i);
        st_elem<ES>(out, i, f2i_decode_one<ES>(k, p, o));
    }
}

unsigned st_grid(uint64_t n)
{
    uint64_t b = (n + ST_THREADS * 8 - 1) / (ST_THREADS * 8);
    uint64_t cap = (uint64_t)sm_count() * 4;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

}  // namespace

unsigned stats_grid(uint64_t n) { return st_grid(n); }

void launch_stats(const uint8_t *in, uint64_t n, int es, Order o, StatsAcc *acc, double *fsum_partial,
                  cudaStream_t s)
{
    GTSC_CUDA(cudaMemsetAsync(acc, 0, sizeof(StatsAcc), s));
    if (n == 0) return;
    const unsigned g = st_grid(n);
    switch (es) {
    case 1: k_stats<1><<<g, ST_THREADS, 0, s>>>(in, n, o, acc, fsum_partial); break;
    case 2: k_stats<2><<<g, ST_THREADS, 0, s>>>(in, n, o, acc, fsum_partial); break;
    case 4: k_stats<4><<<g, ST_THREADS, 0, s>>>(in, n, o, acc, fsum_partial); break;
    default: k_stats<8><<<g, ST_THREADS, 0, s>>>(in, n, o, acc, fsum_partial); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_log_table(int *table, cudaStream_t s)
{
    k_log_table<<<1, 32, 0, s>>>(table);
    GTSC_CUDA(cudaGetLastError());
}

void launch_f2i_encode(const uint8_t *in, uint64_t n, int es, Order o, int p, int32_t *out, unsigned int *lossy,
                       cudaStream_t s)
{
    if (n == 0) return;
    const unsigned g = st_grid(n);
    switch (es) {
    case 1: k_f2i_encode<1><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out, lossy); break;
    case 2: k_f2i_encode<2><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out, lossy); break;
    case 4: k_f2i_encode<4><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out, lossy); break;
    default: k_f2i_encode<8><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out, lossy); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_f2i_decode(const uint8_t *in, uint64_t n, int es, Order o, int p, uint8_t *out, cudaStream_t s)
{
    if (n == 0) return;
    const unsigned g = st_grid(n);
    switch (es) {
    case 1: k_f2i_decode<1><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out); break;
    case 2: k_f2i_decode<2><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out); break;
    case 4: k_f2i_decode<4><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out); break;
    default: k_f2i_decode<8><<<g, ST_THREADS, 0, s>>>(in, n, o, p, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
