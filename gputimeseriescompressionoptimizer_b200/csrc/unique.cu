// unique.cu -- the standalone UniqueEncoding (compression/unique/unique_encoding.cu:35-46, 133-181,
// 261-304): metadata = size_t uniqueCnt, size_t n, T table[uniqueCnt] (the distinct values in
// ascending order); data = uint32 words holding 32/bits codes each (bits = ALT_BITLEN(uniqueCnt-1),
// code of element i at bits [bits*(i%per), ...) of word i/per), where code = the value's table index.
//
// Distinct values: an LSD radix sort of the elements' order keys (32-bit keys for types of up to 4
// bytes, 64-bit otherwise; 8-bit digits), then an adjacent-difference compaction.  A sort pass is
//   1. k_rcount: per 4096-key tile, a shared-memory count of each digit -> counts[digit][tile];
//   2. an inclusive scan over counts in (digit, tile) order;
//   3. k_rscatter: a stable scatter; within a tile, warp w owns keys [512w, 512w + 512) and walks
//      them 32 at a time, ranking equal digits with __match_any_sync and a per-(warp, digit) counter.
// Codes are lower_bound positions in the sorted key table (shared memory when it fits).
//
// Keys are the order keys of the raw bits (IEEE total order for floats), so distinct means distinct
// bit patterns: NaN payloads and signed zeros get their own codes.  The reference sorts with thrust
// and compares with ==, which merges -0.0 into +0.0 and gives every NaN code 0 (lossy); the order of
// the table is the same otherwise.  Code slots past n in the last word are 0 (the reference reads
// past the end of its input there).
#include "encodings.hpp"
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int kRThreads = 256;
constexpr int kRWarps = kRThreads / 32;
constexpr int kRPer = 16;                       // keys per thread
constexpr int kRTile = kRThreads * kRPer;       // 4096 keys per tile
constexpr int kRWarpKeys = 32 * kRPer;          // 512 keys per warp

template <typename K>
__device__ __forceinline__ K key_of(uint64_t u, int es, Order o)
{
    if constexpr (sizeof(K) == 4) {
        if (o == ORD_F32) return (uint32_t)order_key(u, 4, o);
        return (uint32_t)sext(u, es) ^ 0x80000000u;
    } else {
        return order_key(u, 8, o);
    }
}

template <typename K>
__device__ __forceinline__ uint64_t value_of(K k, int es, Order o)
{
    if constexpr (sizeof(K) == 4) {
        if (o == ORD_F32) return order_unkey(k, 4, o);
        const uint64_t s = (uint64_t)(int64_t)(int32_t)(k ^ 0x80000000u);
        return es == 8 ? s : (s & ((1ull << (8 * es)) - 1));
    } else {
        return order_unkey(k, 8, o);
    }
}

template <typename K, int ES>
__global__ void k_ukeys(const uint8_t *__restrict__ in, uint64_t n, Order o, K *__restrict__ keys)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = key_of<K>(ld_elem<ES>(in, i), ES, o);
}

template <typename K>
__global__ void __launch_bounds__(kRThreads) k_rcount(const K *__restrict__ keys, uint64_t n, int shift,
                                                      uint64_t tiles, int32_t *__restrict__ counts)
{
    __shared__ uint32_t hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRTile;
#pragma unroll 4
    for (int j = 0; j < kRPer; j++) {
        const uint64_t i = base + (uint64_t)j * kRThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[(uint32_t)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * tiles + blockIdx.x] = (int32_t)hist[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kRThreads) k_rscatter(const K *__restrict__ keys, uint64_t n, int shift,
                                                        uint64_t tiles, const int32_t *__restrict__ counts,
                                                        const unsigned long long *__restrict__ incl,
                                                        K *__restrict__ out)
{
    __shared__ uint32_t wcnt[kRWarps][256];
    __shared__ unsigned long long gbase[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kRWarps; k++) wcnt[k][threadIdx.x] = 0;
    {
        const uint64_t c = (uint64_t)threadIdx.x * tiles + blockIdx.x;
        gbase[threadIdx.x] = incl[c] - (unsigned long long)counts[c];
    }
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRTile + (uint64_t)w * kRWarpKeys;
    const unsigned lt = (1u << lane) - 1;
    K kv[kRPer];
    uint32_t rk[kRPer];
#pragma unroll
    for (int j = 0; j < kRPer; j++) {
        const uint64_t i = base + (uint64_t)j * 32 + lane;
        const bool valid = i < n;
        kv[j] = valid ? keys[i] : K(0);
        // lanes past the end get a tag no digit has, so they never join a group
        const uint32_t d = valid ? ((uint32_t)(kv[j] >> shift) & 255u) : 256u + lane;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t old = valid ? wcnt[w][d] : 0u;
        rk[j] = old + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[w][d] = old + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {   // exclusive prefix over the warps of each digit
        uint32_t run = 0;
#pragma unroll
        for (int k = 0; k < kRWarps; k++) {
            const uint32_t t = wcnt[k][threadIdx.x];
            wcnt[k][threadIdx.x] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kRPer; j++) {
        const uint64_t i = base + (uint64_t)j * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)(kv[j] >> shift) & 255u;
            out[gbase[d] + wcnt[w][d] + rk[j]] = kv[j];
        }
    }
}

template <typename K>
__global__ void k_uflags(const K *__restrict__ keys, uint64_t n, int32_t *__restrict__ flags)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

template <typename K>
__global__ void k_ucompact(const K *__restrict__ keys, uint64_t n, const int32_t *__restrict__ flags,
                           const unsigned long long *__restrict__ incl, K *__restrict__ table)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (flags[i]) table[incl[i] - 1] = keys[i];
}

// metadata: sizes, then the table values
template <typename K, int ES>
__global__ void k_umeta(const K *__restrict__ table, const unsigned long long *__restrict__ m_p, uint64_t n,
                        Order o, uint8_t *__restrict__ meta)
{
    const uint64_t m = *m_p;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        ((unsigned long long *)meta)[0] = m;
        ((unsigned long long *)meta)[1] = n;
    }
    for (uint64_t j = t; j < m; j += (uint64_t)gridDim.x * blockDim.x)
        st_elem<ES>(meta + 16, j, value_of<K>(table[j], ES, o));
}

template <typename K>
__device__ __forceinline__ uint32_t lower_bound(const K *t, uint32_t m, K key)
{
    uint32_t lo = 0, hi = m;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (t[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// one thread per output word; the table sits in shared memory when SMEM
template <typename K, int ES, bool SMEM>
__global__ void k_ucodes(const uint8_t *__restrict__ in, uint64_t n, Order o, const K *__restrict__ table,
                         uint32_t m, int bits, int per, uint64_t words, uint32_t *__restrict__ out)
{
    extern __shared__ __align__(16) uint8_t u_smem[];
    const K *tab = table;
    if constexpr (SMEM) {
        K *st = (K *)u_smem;
        for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) st[j] = table[j];
        __syncthreads();
        tab = st;
    }
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t acc = 0;
        const uint64_t first = w * per;
        for (int i = 0; i < per; i++) {
            const uint64_t idx = first + i;
            if (idx >= n) break;
            const K k = key_of<K>(ld_elem<ES>(in, idx), ES, o);
            acc |= lower_bound<K>(tab, m, k) << (bits * i);
        }
        out[w] = acc;
    }
}

// one thread per word; codes at or past the table size are corrupt input (value 0, error flag)
template <int ES, bool ALIGNED>
__global__ void k_udecode(const uint8_t *__restrict__ words, uint64_t nwords, const uint8_t *__restrict__ table,
                          uint64_t m, uint64_t n, int bits, int per, uint8_t *__restrict__ out,
                          uint32_t *__restrict__ error)
{
    const uint32_t mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1);
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t word = ALIGNED ? __ldg((const uint32_t *)words + w) : (uint32_t)ld_unaligned<4>(words + 4 * w);
        const uint64_t first = w * per;
        for (int i = 0; i < per; i++) {
            const uint64_t idx = first + i;
            if (idx >= n) break;
            const uint32_t code = (word >> (bits * i)) & mask;
            uint64_t v = 0;
            if (code < m) v = ld_unaligned<ES>(table + (uint64_t)code * ES);
            else atomicOr(error, 1u);
            st_elem<ES>(out, idx, v);
        }
    }
}

int alt_bitlen(uint64_t v)
{
    if ((int64_t)v < 0 || v > 0x7fffffffull) return 32;
    int r = 0;
    while (v >> 1) { v >>= 1; r++; }
    return r + 1;
}

unsigned grid_for(uint64_t items, int threads = 256)
{
    const uint64_t b = (items + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sm_count() * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

// the sorted distinct keys of in[0..n): returns the table (device keys) and m
template <typename K, int ES>
DevBuf distinct_sorted(const uint8_t *in, uint64_t n, Order o, uint64_t *m_out, DevBuf *m_dev, cudaStream_t s)
{
    const uint64_t tiles = (n + kRTile - 1) / kRTile;
    DevBuf a = dev_alloc(n * sizeof(K), s), b = dev_alloc(n * sizeof(K), s);
    k_ukeys<K, ES><<<grid_for(n), 256, 0, s>>>(in, n, o, (K *)a.get());
    GTSC_CUDA(cudaGetLastError());
    const uint64_t nc = 256 * tiles;
    const uint64_t big = std::max(nc, n);
    DevBuf counts = dev_alloc(std::max(nc, n) * 4, s);            // digit counts, later the flags
    DevBuf incl = dev_alloc(big * 8, s);
    DevBuf scratch = dev_alloc(lookback_bytes(rle_tiles(big)), s);
    for (int shift = 0; shift < 8 * (int)sizeof(K); shift += 8) {
        k_rcount<K><<<(unsigned)tiles, kRThreads, 0, s>>>((const K *)a.get(), n, shift, tiles, (int32_t *)counts.get());
        GTSC_CUDA(cudaGetLastError());
        launch_scan_i32(counts.get(), nc, (unsigned long long *)incl.get(), scratch.get(), s);
        k_rscatter<K><<<(unsigned)tiles, kRThreads, 0, s>>>((const K *)a.get(), n, shift, tiles,
                                                          (const int32_t *)counts.get(),
                                                          (const unsigned long long *)incl.get(), (K *)b.get());
        GTSC_CUDA(cudaGetLastError());
        std::swap(a, b);
    }
    k_uflags<K><<<grid_for(n), 256, 0, s>>>((const K *)a.get(), n, (int32_t *)counts.get());
    GTSC_CUDA(cudaGetLastError());
    launch_scan_i32(counts.get(), n, (unsigned long long *)incl.get(), scratch.get(), s);
    k_ucompact<K><<<grid_for(n), 256, 0, s>>>((const K *)a.get(), n, (const int32_t *)counts.get(),
                                              (const unsigned long long *)incl.get(), (K *)b.get());
    GTSC_CUDA(cudaGetLastError());
    *m_dev = dev_alloc(8, s);
    GTSC_CUDA(cudaMemcpyAsync(m_dev->get(), incl.get() + (n - 1) * 8, 8, cudaMemcpyDeviceToDevice, s));
    unsigned long long m = 0;
    d2h(&m, m_dev->get(), 8, s);
    *m_out = m;
    return b;
}

template <typename K, int ES>
Parts unique_encode_t(int dt, View in, cudaStream_t s)
{
    const Order o = native_order(dt);
    const uint64_t n = in.bytes / ES;
    uint64_t m = 0;
    DevBuf m_dev;
    DevBuf table = distinct_sorted<K, ES>(in.ptr, n, o, &m, &m_dev, s);
    const int bits = alt_bitlen(m - 1);
    const int per = 32 / bits;
    const uint64_t words = (n + per - 1) / per;
    Parts r(2);
    r[0] = dev_alloc(16 + m * ES, s);
    r[1] = dev_alloc(words * 4, s);
    k_umeta<K, ES><<<grid_for(m), 256, 0, s>>>((const K *)table.get(), (const unsigned long long *)m_dev.get(), n, o,
                                              r[0].get());
    GTSC_CUDA(cudaGetLastError());
    const uint64_t tb = m * sizeof(K);
    if (tb <= 96 * 1024) {
        auto kern = k_ucodes<K, ES, true>;
        GTSC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        kern<<<grid_for(words), 256, tb, s>>>(in.ptr, n, o, (const K *)table.get(), (uint32_t)m, bits, per, words,
                                             (uint32_t *)r[1].get());
    } else {
        k_ucodes<K, ES, false><<<grid_for(words), 256, 0, s>>>(in.ptr, n, o, (const K *)table.get(), (uint32_t)m, bits,
                                                              per, words, (uint32_t *)r[1].get());
    }
    GTSC_CUDA(cudaGetLastError());
    GTSC_CUDA(cudaStreamSynchronize(s));  // `table` and the scratch die here
    return r;
}

template <int ES>
void launch_udecode(const uint8_t *words, uint64_t nwords, const uint8_t *table, uint64_t m, uint64_t n, int bits,
                    int per, uint8_t *out, uint32_t *err, cudaStream_t s)
{
    const unsigned g = grid_for(nwords);
    if (((uintptr_t)words & 3) == 0) k_udecode<ES, true><<<g, 256, 0, s>>>(words, nwords, table, m, n, bits, per, out, err);
    else k_udecode<ES, false><<<g, 256, 0, s>>>(words, nwords, table, m, n, bits, per, out, err);
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace

Parts unique_encode(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (in.bytes % es) fail(GTSC_ERR_ARG, "unique: input is not a whole number of elements");
    if (in.bytes == 0) return Parts{dev_alloc(0, s), dev_alloc(0, s)};
    if (((uintptr_t)in.ptr) % es) fail(GTSC_ERR_ARG, "unique: input must be element aligned");
    if (in.bytes / es > 0x7fffffffull) fail(GTSC_ERR_ARG, "unique: at most 2^31 - 1 elements");
    switch (es) {
    case 1: return unique_encode_t<uint32_t, 1>(dt, in, s);
    case 2: return unique_encode_t<uint32_t, 2>(dt, in, s);
    case 4: return unique_encode_t<uint32_t, 4>(dt, in, s);
    default: return unique_encode_t<unsigned long long, 8>(dt, in, s);
    }
}

uint64_t unique_count(int dt, View in, cudaStream_t s)
{
    const int es = dtype_size(dt);
    const uint64_t n = in.bytes / es;
    if (n == 0) return 0;
    if (((uintptr_t)in.ptr) % es) fail(GTSC_ERR_ARG, "unique: input must be element aligned");
    if (n > 0x7fffffffull) fail(GTSC_ERR_ARG, "unique: at most 2^31 - 1 elements");
    uint64_t m = 0;
    DevBuf m_dev, t;
    const Order o = native_order(dt);
    switch (es) {
    case 1: t = distinct_sorted<uint32_t, 1>(in.ptr, n, o, &m, &m_dev, s); break;
    case 2: t = distinct_sorted<uint32_t, 2>(in.ptr, n, o, &m, &m_dev, s); break;
    case 4: t = distinct_sorted<uint32_t, 4>(in.ptr, n, o, &m, &m_dev, s); break;
    default: t = distinct_sorted<unsigned long long, 8>(in.ptr, n, o, &m, &m_dev, s); break;
    }
    return m;
}

DevBuf unique_decode(int dt, View meta, View data, cudaStream_t s)
{
    const int es = dtype_size(dt);
    if (data.bytes == 0) return dev_alloc(0, s);
    if (meta.bytes < 16) fail(GTSC_ERR_FORMAT, "unique: metadata too short");
    unsigned long long sz[2];
    d2h(sz, meta.ptr, 16, s);
    const uint64_t m = sz[0], n = sz[1];
    if (m == 0 || m > 0x7fffffffull || 16 + m * es > meta.bytes) fail(GTSC_ERR_FORMAT, "unique: bad table size");
    const int bits = alt_bitlen(m - 1);
    const int per = 32 / bits;
    if (n > (data.bytes / 4) * (uint64_t)per) fail(GTSC_ERR_FORMAT, "unique: code words missing");
    const uint64_t words = (n + per - 1) / per;
    DevBuf out = dev_alloc(n * es, s);
    DevBuf err = dev_alloc(4, s);
    GTSC_CUDA(cudaMemsetAsync(err.get(), 0, 4, s));
    switch (es) {
    case 1: launch_udecode<1>(data.ptr, words, meta.ptr + 16, m, n, bits, per, out.get(), (uint32_t *)err.get(), s); break;
    case 2: launch_udecode<2>(data.ptr, words, meta.ptr + 16, m, n, bits, per, out.get(), (uint32_t *)err.get(), s); break;
    case 4: launch_udecode<4>(data.ptr, words, meta.ptr + 16, m, n, bits, per, out.get(), (uint32_t *)err.get(), s); break;
    default: launch_udecode<8>(data.ptr, words, meta.ptr + 16, m, n, bits, per, out.get(), (uint32_t *)err.get(), s); break;
    }
    uint32_t e = 0;
    d2h(&e, err.get(), 4, s);
    if (e) fail(GTSC_ERR_FORMAT, "unique: code outside the table");
    return out;
}

}  // namespace gtsc
