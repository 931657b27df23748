// learned.cu -- the learned tree planner (see learned.hpp): the feature kernel, the MLP's forward,
// backward and Adam kernels (FP32, deterministic reductions: every sum runs in a fixed order, so a
// gradient is reproducible bit for bit), and the host side of training and inference.
#include "learned.hpp"
#include "vec.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

namespace gtsc {

namespace {

// ------------------------------------------------------------------------------- features
struct FeatDev {
    const uint8_t *data;
    uint64_t n_total;
    uint32_t m;        // sample elements
    int32_t dtype;
};

__device__ __forceinline__ int bits_of(uint64_t v) { return v ? 64 - __clzll((long long)v) : 0; }
__device__ __forceinline__ Order feat_order(int dt)
{
    return dt == GTSC_FLOAT ? ORD_F32 : dt == GTSC_DOUBLE ? ORD_F64 : ORD_INT;
}
__device__ __forceinline__ uint64_t feat_wrap(uint64_t v, int es) { return es == 8 ? v : v & ((1ull << (8 * es)) - 1); }

__device__ __forceinline__ int feat_precision_steps(float x)
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
__device__ __forceinline__ double feat_as_double(uint64_t u, Order o)
{
    if (o == ORD_F32) return (double)__uint_as_float((uint32_t)u);
    if (o == ORD_F64) return __longlong_as_double((long long)u);
    return (double)sext(u, ES);
}

// block-wide reductions over kFeatureThreads threads (fixed order: warp shuffles, then warp 0)
template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T *ws)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T w = ws[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = op(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (lane == 0) ws[0] = w;
    }
    __syncthreads();
    const T r = ws[0];
    __syncthreads();
    return r;
}

struct Top4 {
    uint32_t v[4];
};
__device__ __forceinline__ void top4_push(Top4 &t, uint32_t x)
{
    if (x <= t.v[3]) return;
    t.v[3] = x;
#pragma unroll
    for (int i = 3; i > 0; i--)
        if (t.v[i] > t.v[i - 1]) { const uint32_t y = t.v[i]; t.v[i] = t.v[i - 1]; t.v[i - 1] = y; }
}

// One block per column.  Pass A reads the sample in order (runs, deltas, precision); pass B sorts
// the order keys in shared memory (bitonic) for the value distribution (distinct values, the
// largest multiplicities, percentiles).  Feature definitions are listed in feature_names().
template <int ES>
__global__ void __launch_bounds__(kFeatureThreads) k_features(const FeatDev *cols, float *out)
{
    extern __shared__ __align__(16) unsigned char fsm[];
    unsigned long long *keys = (unsigned long long *)fsm;                 // kFeatureSortCap
    uint32_t *starts = (uint32_t *)(fsm + 8 * kFeatureSortCap);           // kFeatureSortCap
    __shared__ unsigned long long ws64[32];
    __shared__ double wsd[32];
    __shared__ uint32_t ws32[32];
    const FeatDev c = cols[blockIdx.x];
    const Order o = feat_order(c.dtype);
    const uint32_t m = c.m;
    const uint8_t *x = c.data;
    float *f = out + (size_t)blockIdx.x * kFeatures;
    const int W = 8 * ES;
    const bool fp = o != ORD_INT;

    // ---------------- pass A
    uint32_t n_nan = 0, n_inf = 0, unsorted = 0, same = 0, dneg = 0, dd_same = 0, integral = 0;
    unsigned long long kmin = ~0ull, kmax = 0;
    long long dmin = LLONG_MAX, dmax = LLONG_MIN;
    int steps = 0;
    float dbits = 0.f, xbytes = 0.f, d2bits = 0.f;
    for (uint32_t i = threadIdx.x; i < m; i += kFeatureThreads) {
        const uint64_t u = ld_elem<ES>(x, i);
        const bool nan = is_nan_bits(u, o);
        if (fp) {
            n_nan += nan;
            const bool inf = !nan && ((o == ORD_F32) ? ((u >> 23) & 0xff) == 0xff : ((u >> 52) & 0x7ff) == 0x7ff);
            n_inf += inf;
            const double dv = feat_as_double<ES>(u, o);
            integral += (!nan && !inf && dv == rint(dv));
            const float fv = o == ORD_F32 ? __uint_as_float((uint32_t)u) : __double2float_rn(dv);
            const int s = feat_precision_steps(fv);
            steps = s > steps ? s : steps;
        } else {
            integral += 1;
        }
        if (!nan) {
            const unsigned long long k = order_key(u, ES, o);
            kmin = k < kmin ? k : kmin;
            kmax = k > kmax ? k : kmax;
        }
        if (i >= 1) {
            const uint64_t p = ld_elem<ES>(x, i - 1);
            same += (u == p);
            unsorted += lt_native(u, p, ES, o);
            const long long d = sext(u - p, ES);
            dmin = d < dmin ? d : dmin;
            dmax = d > dmax ? d : dmax;
            dneg += d < 0;
            const uint64_t ad = d < 0 ? (uint64_t)(-(d + 1)) + 1 : (uint64_t)d;
            dbits += (float)bits_of(ad);
            xbytes += (float)((bits_of(feat_wrap(u ^ p, ES)) + 7) / 8);
            if (i >= 2) {
                const uint64_t q = ld_elem<ES>(x, i - 2);
                const long long d0 = sext(p - q, ES);
                const long long d2 = sext((uint64_t)d - (uint64_t)d0, ES);
                dd_same += d2 == 0;
                const uint64_t a2 = d2 < 0 ? (uint64_t)(-(d2 + 1)) + 1 : (uint64_t)d2;
                d2bits += (float)bits_of(a2);
            }
        }
    }
    auto add32 = [](uint32_t a, uint32_t b) { return a + b; };
    auto addf = [](double a, double b) { return a + b; };
    n_nan = block_reduce<uint32_t>(n_nan, add32, ws32);
    n_inf = block_reduce<uint32_t>(n_inf, add32, ws32);
    unsorted = block_reduce<uint32_t>(unsorted, add32, ws32);
    same = block_reduce<uint32_t>(same, add32, ws32);
    dneg = block_reduce<uint32_t>(dneg, add32, ws32);
    dd_same = block_reduce<uint32_t>(dd_same, add32, ws32);
    integral = block_reduce<uint32_t>(integral, add32, ws32);
    steps = (int)block_reduce<uint32_t>((uint32_t)steps, [](uint32_t a, uint32_t b) { return a > b ? a : b; }, ws32);
    kmin = block_reduce<unsigned long long>(kmin, [](unsigned long long a, unsigned long long b) { return a < b ? a : b; }, ws64);
    kmax = block_reduce<unsigned long long>(kmax, [](unsigned long long a, unsigned long long b) { return a > b ? a : b; }, ws64);
    dmin = (long long)block_reduce<unsigned long long>((unsigned long long)dmin, [](unsigned long long a, unsigned long long b) {
        return (long long)a < (long long)b ? a : b; }, ws64);
    dmax = (long long)block_reduce<unsigned long long>((unsigned long long)dmax, [](unsigned long long a, unsigned long long b) {
        return (long long)a > (long long)b ? a : b; }, ws64);
    const double sdb = block_reduce<double>((double)dbits, addf, wsd);
    const double sxb = block_reduce<double>((double)xbytes, addf, wsd);
    const double sd2 = block_reduce<double>((double)d2bits, addf, wsd);

    // ---------------- pass B: sort the keys (NaNs included, at their twiddled positions)
    uint32_t P = 1;
    while (P < m) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += kFeatureThreads)
        keys[i] = i < m ? order_key(ld_elem<ES>(x, i), ES, o) : ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += kFeatureThreads) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = keys[i], b = keys[l];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // run starts in sorted order: starts[i] = the first index of i's value (inclusive max-scan)
    constexpr uint32_t PER = kFeatureSortCap / kFeatureThreads;
    const uint32_t c0 = threadIdx.x * PER;
    uint32_t run_max = 0, distinct = 0;
    for (uint32_t q = 0; q < PER; q++) {
        const uint32_t i = c0 + q;
        if (i < m && (i == 0 || keys[i] != keys[i - 1])) {
            run_max = i;
            ++distinct;
        }
    }
    // exclusive max over the threads before this one
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t v = run_max;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v = v > y ? v : y;
        }
        if (lane == 31) ws32[warp] = v;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = ws32[lane];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w = w > y ? w : y;
            }
            ws32[lane] = w;
        }
        __syncthreads();
        const uint32_t before_warp = warp ? ws32[warp - 1] : 0u;
        const uint32_t before_lane = __shfl_up_sync(0xffffffffu, v, 1);
        uint32_t run = lane ? (before_lane > before_warp ? before_lane : before_warp) : before_warp;
        for (uint32_t q = 0; q < PER; q++) {
            const uint32_t i = c0 + q;
            if (i < m && (i == 0 || keys[i] != keys[i - 1])) run = i;
            starts[i] = run;
        }
        __syncthreads();
    }
    distinct = block_reduce<uint32_t>(distinct, add32, ws32);
    Top4 t4{{0, 0, 0, 0}};
    for (uint32_t q = 0; q < PER; q++) {
        const uint32_t i = c0 + q;
        if (i < m && (i + 1 == m || keys[i + 1] != keys[i])) top4_push(t4, i - starts[i] + 1);
    }
    // merge the threads' top-4 lists: warps by shuffles, then warp 0 over the warps
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            Top4 other;
#pragma unroll
            for (int j = 0; j < 4; j++) other.v[j] = __shfl_xor_sync(0xffffffffu, t4.v[j], off);
#pragma unroll
            for (int j = 0; j < 4; j++) top4_push(t4, other.v[j]);
        }
        __syncthreads();
        uint32_t *tw = starts;  // reuse: 32 warps x 4
        if (lane == 0)
            for (int j = 0; j < 4; j++) tw[warp * 4 + j] = t4.v[j];
        __syncthreads();
        if (threadIdx.x == 0) {
            Top4 all{{0, 0, 0, 0}};
            for (int w = 0; w < kFeatureThreads / 32; w++)
                for (int j = 0; j < 4; j++) top4_push(all, tw[w * 4 + j]);
            t4 = all;
        }
    }

    if (threadIdx.x != 0) return;
    for (int j = 0; j < kFeatures; j++) f[j] = 0.f;
    if (c.dtype >= 0 && c.dtype < 6) f[c.dtype] = 1.f;
    f[6] = (float)(log2((double)c.n_total + 1.0) / 32.0);
    f[7] = (float)m / (float)kFeatureSample;
    if (m == 0) return;
    const float fm = (float)m, fm1 = m > 1 ? (float)(m - 1) : 1.f, fm2 = m > 2 ? (float)(m - 2) : 1.f;
    f[8] = n_nan / fm;
    f[9] = n_inf / fm;
    f[10] = unsorted == 0 ? 1.f : 0.f;
    f[11] = m > 1 ? same / fm1 : 0.f;
    const uint32_t runs = m - same;
    f[12] = (float)(log2((double)m / (double)runs) / 14.0);
    f[13] = distinct / fm;
    f[14] = (float)(log2((double)distinct) / 14.0);
    f[15] = t4.v[0] / fm;
    f[16] = (t4.v[0] + t4.v[1] + t4.v[2] + t4.v[3]) / fm;
    const bool any = kmin <= kmax;  // false when every element is NaN
    const uint64_t krange = any ? kmax - kmin : 0;
    if (!fp) {
        const int64_t mn = any ? sext(order_unkey(kmin, ES, o), ES) : 0, mx = any ? sext(order_unkey(kmax, ES, o), ES) : 0;
        f[17] = (float)bitlen_signed(mn, mx, ES) / W;
    } else {
        f[17] = (float)bits_of(krange) / W;
    }
    f[18] = (float)bits_of(krange) / W;
    const unsigned long long kp90 = keys[(uint32_t)(((uint64_t)(m - 1) * 9) / 10)];
    f[19] = (float)bits_of(any && kp90 > kmin ? kp90 - kmin : 0) / W;
    if (any) {
        const unsigned long long tk = kmin + (unsigned long long)((double)krange * 0.9);
        uint32_t lo = 0, hi = m;  // first key >= tk
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (keys[mid] < tk) lo = mid + 1;
            else hi = mid;
        }
        uint32_t lo2 = lo, hi2 = m;  // first key > kmax (NaN keys above the largest number)
        while (lo2 < hi2) {
            const uint32_t mid = (lo2 + hi2) >> 1;
            if (keys[mid] <= kmax) lo2 = mid + 1;
            else hi2 = mid;
        }
        f[20] = (lo2 - lo) / fm;
    }
    if (m > 1) {
        f[21] = (float)bitlen_signed(dmin, dmax, ES) / W;
        f[22] = (float)bits_of((uint64_t)dmax - (uint64_t)dmin) / W;
        f[23] = dneg / fm1;
        f[24] = (float)(sdb / fm1) / W;
        f[25] = (float)(sxb / fm1) / ES;
    }
    if (fp) {
        f[26] = steps / 10.f;
        const double mn = any ? feat_as_double<ES>(order_unkey(kmin, ES, o), o) : 0.0;
        const double mx = any ? feat_as_double<ES>(order_unkey(kmax, ES, o), o) : 0.0;
        double sc = 1.0;
        for (int i = 0; i < steps && i < 10; i++) sc *= 10.0;
        const bool ok = steps < 10 && any && n_inf == 0 && mn * sc > -2147483648.0 && mx * sc < 2147483647.0;
        f[27] = ok ? 1.f : 0.f;
        f[28] = ok ? (float)(log2(1.0 + (mx - mn) * sc) / 32.0) : 1.f;
    } else {
        f[28] = (float)bits_of(krange) / 32.f;
    }
    f[29] = integral / fm;
    if (m > 2) {
        f[30] = dd_same / fm2;
        f[31] = (float)(sd2 / fm2) / W;
    }
}

// ------------------------------------------------------------------------------- MLP
// y[b, o] = act(sum_i x[b, i] * W[i, o] + bias[o]); one thread per (b, o), sum over i in order
__global__ void k_linear(const float *x, const float *W, const float *bias, float *y, int B, int I, int O, int relu)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * O) return;
    const int b = t / O, oo = t % O;
    float s = bias[oo];
    for (int i = 0; i < I; i++) s = __fmaf_rn(x[(size_t)b * I + i], W[(size_t)i * O + oo], s);
    y[t] = relu ? fmaxf(s, 0.f) : s;
}

// per row: softmax over the valid classes, loss = -log p[label], dlogits = (p - onehot) / n_valid
__global__ void k_softmax_xent(const float *logits, const int32_t *labels, const uint8_t *mask, float *dlogits,
                               float *row_loss, int B, int K, float inv_n)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float *z = logits + (size_t)b * K;
    const uint8_t *mk = mask + (size_t)b * K;
    float *dz = dlogits + (size_t)b * K;
    const int y = labels[b];
    if (y < 0) {
        for (int k = 0; k < K; k++) dz[k] = 0.f;
        row_loss[b] = 0.f;
        return;
    }
    float mx = -INFINITY;
    for (int k = 0; k < K; k++)
        if (mk[k]) mx = fmaxf(mx, z[k]);
    float sum = 0.f;
    for (int k = 0; k < K; k++)
        if (mk[k]) sum += __expf(z[k] - mx);
    const float lse = mx + __logf(sum);
    for (int k = 0; k < K; k++) {
        const float p = mk[k] ? __expf(z[k] - lse) : 0.f;
        dz[k] = (p - (k == y ? 1.f : 0.f)) * inv_n;
    }
    row_loss[b] = lse - z[y];
}

// dW[i, o] = sum_b x[b, i] * dy[b, o]; db[o] = sum_b dy[b, o]; one thread per (i, o) (+ O for db)
__global__ void k_linear_grad_w(const float *x, const float *dy, float *dW, float *db, int B, int I, int O)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < I * O) {
        const int i = t / O, oo = t % O;
        float s = 0.f;
        for (int b = 0; b < B; b++) s = __fmaf_rn(x[(size_t)b * I + i], dy[(size_t)b * O + oo], s);
        dW[t] = s;
    } else if (t < I * O + O) {
        const int oo = t - I * O;
        float s = 0.f;
        for (int b = 0; b < B; b++) s += dy[(size_t)b * O + oo];
        db[oo] = s;
    }
}

// dx[b, i] = (sum_o dy[b, o] * W[i, o]) * (h[b, i] > 0); h = the layer's ReLU output
__global__ void k_linear_grad_x(const float *dy, const float *W, const float *h, float *dx, int B, int I, int O)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * I) return;
    const int b = t / I, i = t % I;
    float s = 0.f;
    for (int oo = 0; oo < O; oo++) s = __fmaf_rn(dy[(size_t)b * O + oo], W[(size_t)i * O + oo], s);
    dx[t] = h[t] > 0.f ? s : 0.f;
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// rows of x gathered by idx and normalised: xn[r, f] = (x[idx[r], f] - mu[f]) / sd[f]
__global__ void k_gather_norm(const float *x, const int32_t *idx, const float *mu, const float *sd, float *xn, int B)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * kFeatures) return;
    const int r = t / kFeatures, f = t % kFeatures;
    xn[t] = (x[(size_t)idx[r] * kFeatures + f] - mu[f]) / sd[f];
}

unsigned grid_for(size_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ------------------------------------------------------------------------------- host: features
void compute_features(const std::vector<FeatureColumn> &cols, float *d_out, cudaStream_t s)
{
    if (cols.empty()) return;
    std::vector<FeatDev> h(cols.size());
    int es_all = -1;
    for (size_t c = 0; c < cols.size(); c++) {
        const int es = dtype_size(cols[c].dtype);
        if (!es) fail(GTSC_ERR_ARG, "features: unknown data type");
        h[c].data = (const uint8_t *)cols[c].data;
        h[c].n_total = cols[c].n_total;
        h[c].m = (uint32_t)std::min<uint64_t>(cols[c].n_total, kFeatureSample);
        h[c].dtype = cols[c].dtype;
        if (h[c].m && !cols[c].data) fail(GTSC_ERR_ARG, "features: null column");
        es_all = c == 0 ? es : (es_all == es ? es : 0);
    }
    // one launch per element size (columns grouped by size)
    const size_t smem = (size_t)kFeatureSortCap * 12;
    for (int es : {1, 2, 4, 8}) {
        std::vector<FeatDev> g;
        std::vector<size_t> where;
        for (size_t c = 0; c < cols.size(); c++)
            if (dtype_size(cols[c].dtype) == es) {
                g.push_back(h[c]);
                where.push_back(c);
            }
        if (g.empty()) continue;
        DevBuf dg = dev_alloc(g.size() * sizeof(FeatDev), s);
        GTSC_CUDA(cudaMemcpyAsync(dg.get(), g.data(), g.size() * sizeof(FeatDev), cudaMemcpyHostToDevice, s));
        DevBuf tmp = dev_alloc(g.size() * kFeatures * sizeof(float), s);
        switch (es) {
#define GTSC_FEAT(E)                                                                                            \
    case E:                                                                                                     \
        GTSC_CUDA(cudaFuncSetAttribute(k_features<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_features<E><<<(unsigned)g.size(), kFeatureThreads, smem, s>>>((const FeatDev *)dg.get(), (float *)tmp.get()); \
        break;
            GTSC_FEAT(1) GTSC_FEAT(2) GTSC_FEAT(4) GTSC_FEAT(8)
#undef GTSC_FEAT
        }
        GTSC_CUDA(cudaGetLastError());
        if (g.size() == cols.size()) {
            GTSC_CUDA(cudaMemcpyAsync(d_out, tmp.get(), g.size() * kFeatures * 4, cudaMemcpyDeviceToDevice, s));
        } else {
            for (size_t j = 0; j < g.size(); j++)
                GTSC_CUDA(cudaMemcpyAsync(d_out + where[j] * kFeatures, (float *)tmp.get() + j * kFeatures,
                                          kFeatures * 4, cudaMemcpyDeviceToDevice, s));
        }
        GTSC_CUDA(cudaStreamSynchronize(s));  // the tables above are freed on return
    }
    (void)es_all;
}

// ------------------------------------------------------------------------------- host: planner
namespace {

bool node_supported(int enc, int dt)
{
    if (enc == GTSC_AFL && is_fp(dt)) return false;  // AflEncoding's float split is not on this path
    if (enc == GTSC_UNIQUE) return false;
    return true;
}

std::vector<uint8_t> validity(const std::vector<std::vector<int16_t>> &classes)
{
    std::vector<uint8_t> v(classes.size() * 6, 0);
    for (size_t c = 0; c < classes.size(); c++)
        for (int dt = 0; dt < 6; dt++) {
            try {
                Tree t = tree_from_path(classes[c].data(), (int)classes[c].size(), dt);
                bool ok = t.size() == (int)classes[c].size();
                for (int k = 0; k < t.size(); k++) ok = ok && node_supported(t.enc[k], t.dt[k]);
                // a dictionary's code stream, re-read as 8-byte values by its first child, is not
                // always a whole number of them: only none may sit there (as the planners offer)
                for (int k = 0; k + 1 < t.size(); k++)
                    if (t.enc[k] == GTSC_DICT && dtype_size(t.dt[k]) == 8 && t.enc[k + 1] != GTSC_NONE) ok = false;
                v[c * 6 + dt] = ok;
            } catch (const Error &) {
                v[c * 6 + dt] = 0;
            }
        }
    return v;
}

struct Offs {
    size_t w1, b1, w2, b2, w3, b3;
};
Offs offsets(int K)
{
    Offs o;
    o.w1 = 0;
    o.b1 = o.w1 + (size_t)kFeatures * kHidden;
    o.w2 = o.b1 + kHidden;
    o.b2 = o.w2 + (size_t)kHidden * kHidden;
    o.w3 = o.b2 + kHidden;
    o.b3 = o.w3 + (size_t)kHidden * K;
    return o;
}

// device work buffers of one forward / backward over B rows
struct Work {
    DevBuf buf;
    float *xn, *h1, *h2, *z, *dz, *dh2, *dh1, *loss;
    uint8_t *mask;
    int32_t *idx, *lab;
    int B = 0;
    void ensure(int B_, int K, cudaStream_t s)
    {
        if (B_ <= B) return;
        B = B_;
        const size_t f = (size_t)B * (kFeatures + 2 * kHidden + 2 * K + 2 * kHidden + 1);
        buf = dev_alloc(4 * f + (size_t)B * K + 8ull * B + 256, s);
        float *p = (float *)buf.get();
        xn = p; p += (size_t)B * kFeatures;
        h1 = p; p += (size_t)B * kHidden;
        h2 = p; p += (size_t)B * kHidden;
        z = p; p += (size_t)B * K;
        dz = p; p += (size_t)B * K;
        dh2 = p; p += (size_t)B * kHidden;
        dh1 = p; p += (size_t)B * kHidden;
        loss = p; p += B;
        idx = (int32_t *)p;
        lab = idx + B;
        mask = (uint8_t *)(lab + B);
    }
};

}  // namespace

Planner::Planner(const std::vector<std::vector<int16_t>> &cls, uint64_t seed)
{
    if (cls.empty() || cls.size() > (size_t)kMaxClasses) fail(GTSC_ERR_ARG, "planner: 1..256 classes");
    K = (int)cls.size();
    classes = cls;
    valid = validity(classes);
    mu.assign(kFeatures, 0.f);
    sd.assign(kFeatures, 1.f);
    const size_t n = n_params();
    params = dev_alloc(4 * n, nullptr);
    grads = dev_alloc(4 * n, nullptr);
    adam_m = dev_alloc(4 * n, nullptr);
    adam_v = dev_alloc(4 * n, nullptr);
    // He-uniform initialisation from a seeded generator; biases 0
    std::vector<float> h(n, 0.f);
    std::mt19937_64 rng(seed);
    const Offs o = offsets(K);
    auto fill = [&](size_t off, int fan_in, size_t cnt) {
        const float a = std::sqrt(6.f / (float)fan_in);
        std::uniform_real_distribution<float> u(-a, a);
        for (size_t i = 0; i < cnt; i++) h[off + i] = u(rng);
    };
    fill(o.w1, kFeatures, (size_t)kFeatures * kHidden);
    fill(o.w2, kHidden, (size_t)kHidden * kHidden);
    fill(o.w3, kHidden, (size_t)kHidden * K);
    set_params(h.data(), nullptr);
    GTSC_CUDA(cudaMemset(adam_m.get(), 0, 4 * n));
    GTSC_CUDA(cudaMemset(adam_v.get(), 0, 4 * n));
    GTSC_CUDA(cudaDeviceSynchronize());
}

void Planner::set_params(const float *h, cudaStream_t s)
{
    GTSC_CUDA(cudaMemcpyAsync(params.get(), h, 4 * n_params(), cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaStreamSynchronize(s));
}

void Planner::get_params(float *h, cudaStream_t s) const
{
    d2h(h, params.get(), 4 * n_params(), s);
}

namespace {

// forward over B gathered rows (w.idx) into w.z
void run_batch(Planner &P, Work &w, const float *d_x, int B, cudaStream_t s, const float *d_mu, const float *d_sd)
{
    const int K = P.K;
    const Offs o = offsets(K);
    const float *W = (const float *)P.params.get();
    const unsigned bs = 256;
    k_gather_norm<<<grid_for((size_t)B * kFeatures, bs), bs, 0, s>>>(d_x, w.idx, d_mu, d_sd, w.xn, B);
    k_linear<<<grid_for((size_t)B * kHidden, bs), bs, 0, s>>>(w.xn, W + o.w1, W + o.b1, w.h1, B, kFeatures, kHidden, 1);
    k_linear<<<grid_for((size_t)B * kHidden, bs), bs, 0, s>>>(w.h1, W + o.w2, W + o.b2, w.h2, B, kHidden, kHidden, 1);
    k_linear<<<grid_for((size_t)B * K, bs), bs, 0, s>>>(w.h2, W + o.w3, W + o.b3, w.z, B, kHidden, K, 0);
    GTSC_CUDA(cudaGetLastError());
}

void backward_pass(Planner &P, Work &w, int B, cudaStream_t s)
{
    const int K = P.K;
    const Offs o = offsets(K);
    const float *W = (const float *)P.params.get();
    float *G = (float *)P.grads.get();
    const unsigned bs = 256;
    k_linear_grad_w<<<grid_for((size_t)kHidden * K + K, bs), bs, 0, s>>>(w.h2, w.dz, G + o.w3, G + o.b3, B, kHidden, K);
    k_linear_grad_x<<<grid_for((size_t)B * kHidden, bs), bs, 0, s>>>(w.dz, W + o.w3, w.h2, w.dh2, B, kHidden, K);
    k_linear_grad_w<<<grid_for((size_t)kHidden * kHidden + kHidden, bs), bs, 0, s>>>(w.h1, w.dh2, G + o.w2, G + o.b2, B,
                                                                                     kHidden, kHidden);
    k_linear_grad_x<<<grid_for((size_t)B * kHidden, bs), bs, 0, s>>>(w.dh2, W + o.w2, w.h1, w.dh1, B, kHidden, kHidden);
    k_linear_grad_w<<<grid_for((size_t)kFeatures * kHidden + kHidden, bs), bs, 0, s>>>(w.xn, w.dh1, G + o.w1, G + o.b1,
                                                                                       B, kFeatures, kHidden);
    GTSC_CUDA(cudaGetLastError());
}

// row data types from the one-hot features (host copy of the features' first 6 columns)
std::vector<int32_t> row_dtypes(const float *d_x, uint32_t n, cudaStream_t s)
{
    std::vector<float> hx((size_t)n * kFeatures);
    d2h(hx.data(), d_x, hx.size() * 4, s);
    std::vector<int32_t> dt(n, 0);
    for (uint32_t r = 0; r < n; r++)
        for (int k = 0; k < 6; k++)
            if (hx[(size_t)r * kFeatures + k] > 0.5f) dt[r] = k;
    return dt;
}

}  // namespace

float Planner::gradient(const float *d_x, const int32_t *h_labels, uint32_t n, float *h_grad, cudaStream_t s)
{
    if (!n) fail(GTSC_ERR_ARG, "planner: no rows");
    Work w;
    w.ensure((int)n, K, s);
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::vector<int32_t> dts = row_dtypes(d_x, n, s);
    std::vector<uint8_t> mask((size_t)n * K);
    uint32_t valid_rows = 0;
    std::vector<int32_t> lab(h_labels, h_labels + n);
    for (uint32_t r = 0; r < n; r++) {
        for (int k = 0; k < K; k++) mask[(size_t)r * K + k] = valid[(size_t)k * 6 + dts[r]];
        if (lab[r] >= K || (lab[r] >= 0 && !valid[(size_t)lab[r] * 6 + dts[r]])) lab[r] = -1;
        valid_rows += lab[r] >= 0;
    }
    if (!valid_rows) fail(GTSC_ERR_ARG, "planner: no labelled rows");
    GTSC_CUDA(cudaMemcpyAsync(w.idx, idx.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync(w.lab, lab.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync(w.mask, mask.data(), mask.size(), cudaMemcpyHostToDevice, s));
    DevBuf norm = dev_alloc(8 * kFeatures, s);
    GTSC_CUDA(cudaMemcpyAsync(norm.get(), mu.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync((float *)norm.get() + kFeatures, sd.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    run_batch(*this, w, d_x, (int)n, s, (float *)norm.get(), (float *)norm.get() + kFeatures);
    const unsigned bs = 256;
    k_softmax_xent<<<grid_for(n, bs), bs, 0, s>>>(w.z, w.lab, w.mask, w.dz, w.loss, (int)n, K, 1.f / valid_rows);
    GTSC_CUDA(cudaGetLastError());
    backward_pass(*this, w, (int)n, s);
    std::vector<float> rl(n);
    d2h(rl.data(), w.loss, 4ull * n, s);
    if (h_grad) d2h(h_grad, grads.get(), 4 * n_params(), s);
    double L = 0;
    for (float x : rl) L += x;
    return (float)(L / valid_rows);
}

float Planner::train(const float *d_x, const int32_t *h_labels, uint32_t n, int epochs, int batch, float lr,
                     uint64_t seed, cudaStream_t s)
{
    if (!n || batch <= 0 || epochs <= 0) fail(GTSC_ERR_ARG, "planner: bad training arguments");
    // normalisation from the training rows
    std::vector<float> hx((size_t)n * kFeatures);
    d2h(hx.data(), d_x, hx.size() * 4, s);
    for (int f = 0; f < kFeatures; f++) {
        double a = 0, b = 0;
        for (uint32_t r = 0; r < n; r++) a += hx[(size_t)r * kFeatures + f];
        a /= n;
        for (uint32_t r = 0; r < n; r++) {
            const double d = hx[(size_t)r * kFeatures + f] - a;
            b += d * d;
        }
        b = std::sqrt(b / n);
        mu[f] = (float)a;
        sd[f] = b > 1e-6 ? (float)b : 1.f;
    }
    std::vector<int32_t> dts(n, 0);
    for (uint32_t r = 0; r < n; r++)
        for (int k = 0; k < 6; k++)
            if (hx[(size_t)r * kFeatures + k] > 0.5f) dts[r] = k;
    std::vector<int32_t> rows;
    for (uint32_t r = 0; r < n; r++)
        if (h_labels[r] >= 0 && h_labels[r] < K && valid[(size_t)h_labels[r] * 6 + dts[r]]) rows.push_back((int32_t)r);
    if (rows.empty()) fail(GTSC_ERR_ARG, "planner: no labelled rows");
    DevBuf norm = dev_alloc(8 * kFeatures, s);
    GTSC_CUDA(cudaMemcpyAsync(norm.get(), mu.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync((float *)norm.get() + kFeatures, sd.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    const float *d_mu = (float *)norm.get(), *d_sd = d_mu + kFeatures;
    const int B = std::min<int>(batch, (int)rows.size());
    Work w;
    w.ensure(B, K, s);
    std::mt19937_64 rng(seed);
    std::vector<int32_t> lab(B);
    std::vector<uint8_t> mask((size_t)B * K);
    const int n_par = (int)n_params();
    const unsigned bs = 256;
    double last = 0;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(rows.begin(), rows.end(), rng);
        double ep_loss = 0;
        int ep_rows = 0;
        for (size_t start = 0; start + B <= rows.size(); start += B) {
            for (int r = 0; r < B; r++) {
                const int row = rows[start + r];
                lab[r] = h_labels[row];
                for (int k = 0; k < K; k++) mask[(size_t)r * K + k] = valid[(size_t)k * 6 + dts[row]];
            }
            GTSC_CUDA(cudaMemcpyAsync(w.idx, rows.data() + start, 4ull * B, cudaMemcpyHostToDevice, s));
            GTSC_CUDA(cudaMemcpyAsync(w.lab, lab.data(), 4ull * B, cudaMemcpyHostToDevice, s));
            GTSC_CUDA(cudaMemcpyAsync(w.mask, mask.data(), mask.size(), cudaMemcpyHostToDevice, s));
            run_batch(*this, w, d_x, B, s, d_mu, d_sd);
            k_softmax_xent<<<grid_for(B, bs), bs, 0, s>>>(w.z, w.lab, w.mask, w.dz, w.loss, B, K, 1.f / B);
            backward_pass(*this, w, B, s);
            ++adam_t;
            const float c1 = 1.f - std::pow(0.9f, (float)adam_t), c2 = 1.f - std::pow(0.999f, (float)adam_t);
            k_adam<<<grid_for(n_par, bs), bs, 0, s>>>((float *)params.get(), (const float *)grads.get(),
                                                     (float *)adam_m.get(), (float *)adam_v.get(), n_par, lr, 0.9f,
                                                     0.999f, 1e-8f, c1, c2);
            GTSC_CUDA(cudaGetLastError());
            if (ep == epochs - 1) {
                std::vector<float> rl(B);
                d2h(rl.data(), w.loss, 4ull * B, s);  // the host vectors above are reused next batch
                for (float x : rl) ep_loss += x;
                ep_rows += B;
            } else {
                GTSC_CUDA(cudaStreamSynchronize(s));
            }
        }
        if (ep == epochs - 1) last = ep_rows ? ep_loss / ep_rows : 0;
    }
    return (float)last;
}

void Planner::predict(const float *d_x, const int32_t *h_dtypes, uint32_t n, int32_t *h_class, float *h_conf,
                      cudaStream_t s)
{
    if (!n) return;
    Work w;
    w.ensure((int)n, K, s);
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    GTSC_CUDA(cudaMemcpyAsync(w.idx, idx.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    DevBuf norm = dev_alloc(8 * kFeatures, s);
    GTSC_CUDA(cudaMemcpyAsync(norm.get(), mu.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    GTSC_CUDA(cudaMemcpyAsync((float *)norm.get() + kFeatures, sd.data(), 4 * kFeatures, cudaMemcpyHostToDevice, s));
    run_batch(*this, w, d_x, (int)n, s, (float *)norm.get(), (float *)norm.get() + kFeatures);
    std::vector<float> z((size_t)n * K);
    d2h(z.data(), w.z, 4 * z.size(), s);
    for (uint32_t r = 0; r < n; r++) {
        const int dt = h_dtypes[r];
        if (dt < 0 || dt >= 6) fail(GTSC_ERR_ARG, "planner: unknown data type");
        float mx = -INFINITY;
        int best = -1;
        for (int k = 0; k < K; k++)
            if (valid[(size_t)k * 6 + dt] && z[(size_t)r * K + k] > mx) {
                mx = z[(size_t)r * K + k];
                best = k;
            }
        float sum = 0.f;
        for (int k = 0; k < K; k++)
            if (valid[(size_t)k * 6 + dt]) sum += std::exp(z[(size_t)r * K + k] - mx);
        h_class[r] = best;
        h_conf[r] = best >= 0 ? 1.f / sum : 0.f;
    }
}

Tree Planner::class_tree(int c, int dtype) const
{
    if (c < 0 || c >= K || !valid[(size_t)c * 6 + dtype]) fail(GTSC_ERR_ARG, "planner: class not valid for the type");
    return tree_from_path(classes[c].data(), (int)classes[c].size(), dtype);
}

// model file: "GTSCMLP1", int32 K, int32 features, int32 hidden, mu[32], sd[32], parameters, then per
// class int32 length + int16 encodings
std::vector<uint8_t> Planner::save() const
{
    std::vector<uint8_t> out;
    auto put = [&](const void *p, size_t n) {
        const uint8_t *b = (const uint8_t *)p;
        out.insert(out.end(), b, b + n);
    };
    put("GTSCMLP1", 8);
    const int32_t hdr[3] = {K, kFeatures, kHidden};
    put(hdr, sizeof hdr);
    put(mu.data(), 4 * kFeatures);
    put(sd.data(), 4 * kFeatures);
    std::vector<float> p(n_params());
    get_params(p.data(), nullptr);
    put(p.data(), 4 * p.size());
    for (const auto &c : classes) {
        const int32_t len = (int32_t)c.size();
        put(&len, 4);
        put(c.data(), 2 * c.size());
    }
    return out;
}

Planner *Planner::load(const void *bytes, uint64_t size)
{
    const uint8_t *b = (const uint8_t *)bytes;
    uint64_t pos = 0;
    auto get = [&](void *dst, uint64_t n) {
        if (pos + n > size) fail(GTSC_ERR_FORMAT, "planner model: truncated");
        std::memcpy(dst, b + pos, n);
        pos += n;
    };
    char magic[8];
    get(magic, 8);
    if (std::memcmp(magic, "GTSCMLP1", 8) != 0) fail(GTSC_ERR_FORMAT, "planner model: bad magic");
    int32_t hdr[3];
    get(hdr, sizeof hdr);
    if (hdr[0] <= 0 || hdr[0] > kMaxClasses || hdr[1] != kFeatures || hdr[2] != kHidden)
        fail(GTSC_ERR_FORMAT, "planner model: unexpected shape");
    const int K = hdr[0];
    std::vector<float> mu(kFeatures), sd(kFeatures), p(mlp_param_count(K));
    get(mu.data(), 4 * kFeatures);
    get(sd.data(), 4 * kFeatures);
    get(p.data(), 4 * p.size());
    std::vector<std::vector<int16_t>> cls(K);
    for (int c = 0; c < K; c++) {
        int32_t len;
        get(&len, 4);
        if (len <= 0 || len > 1024) fail(GTSC_ERR_FORMAT, "planner model: bad class");
        cls[c].resize(len);
        get(cls[c].data(), 2ull * len);
    }
    std::unique_ptr<Planner> P(new Planner(cls, 0));
    P->mu = mu;
    P->sd = sd;
    P->set_params(p.data(), nullptr);
    return P.release();
}

}  // namespace gtsc
