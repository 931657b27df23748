// rle.cu -- run-length encoding (RleEncoding, compression/rle/rle_encode.cu:18-62 and
// rle_decode.cu:19-73) and the generic inclusive scan it and GFC use.
//
// Encode: the reference copies the column into Thrust vectors and runs reduce_by_key, then copies
// the results out.  Here one pass marks run heads (value differs from its left neighbour), ranks
// them with a block scan + decoupled look-back, and writes each run's value and start index;
// a second, run-sized pass turns starts into lengths.
// Decode: inclusive scan of the lengths (run ends), then every thread expands 8 consecutive output
// positions, locating their run by binary search inside the run range of its tile.
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int R_THREADS = 256;
constexpr int R_PER = 8;
constexpr int R_TILE = R_THREADS * R_PER;

__device__ __forceinline__ bool same_val(uint64_t a, uint64_t b, Order o) { return a == b && !is_nan_bits(a, o); }

template <int ES>
__global__ void __launch_bounds__(R_THREADS)
k_rle_heads(const uint8_t *__restrict__ in, uint64_t n, Order o, uint8_t *__restrict__ values,
            uint32_t *__restrict__ starts, unsigned long long *runs_out, Lookback lb)
{
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = claim_tile(lb);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * R_TILE + (uint64_t)threadIdx.x * R_PER;
    uint64_t v[R_PER + 1];
    v[0] = base > 0 && base - 1 < n ? ld_elem<ES>(in, base - 1) : 0;
#pragma unroll
    for (int j = 0; j < R_PER; j++) v[j + 1] = base + j < n ? ld_elem<ES>(in, base + j) : 0;
    uint32_t heads = 0;
#pragma unroll
    for (int j = 0; j < R_PER; j++) {
        const uint64_t i = base + j;
        if (i < n && (i == 0 || !same_val(v[j + 1], v[j], o))) heads |= 1u << j;
    }
    unsigned long long total;
    unsigned long long excl = block_exclusive_scan<R_THREADS>((unsigned long long)__popc(heads), ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    uint64_t r = s_prefix + excl;
    for (int j = 0; j < R_PER; j++)
        if ((heads >> j) & 1u) {
            st_elem<ES>(values, r, v[j + 1]);
            starts[r] = (uint32_t)(base + j);
            ++r;
        }
    if (base < n && base + R_PER >= n) *runs_out = r;
}

__global__ void k_rle_lengths(const uint32_t *__restrict__ starts, const unsigned long long *runs_p, uint64_t n,
                              int32_t *__restrict__ lengths)
{
    const uint64_t runs = *runs_p;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += stride) {
        const uint64_t next = r + 1 < runs ? starts[r + 1] : n;
        lengths[r] = (int32_t)(next - starts[r]);
    }
}

// inclusive scan of int32 (any alignment) into uint64
__global__ void __launch_bounds__(R_THREADS)
k_scan_i32(const uint8_t *__restrict__ in, uint64_t n, unsigned long long *__restrict__ out, Lookback lb)
{
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = claim_tile(lb);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * R_TILE + (uint64_t)threadIdx.x * R_PER;
    long long v[R_PER];
    unsigned long long local = 0;
#pragma unroll
    for (int j = 0; j < R_PER; j++) {
        v[j] = base + j < n ? (long long)(int32_t)ld_unaligned<4>(in + 4 * (base + j)) : 0;
        local += (unsigned long long)v[j];
    }
    unsigned long long total;
    unsigned long long excl = block_exclusive_scan<R_THREADS>(local, ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    unsigned long long acc = s_prefix + excl;
#pragma unroll
    for (int j = 0; j < R_PER; j++) {
        acc += (unsigned long long)v[j];
        if (base + j < n) out[base + j] = acc;
    }
}

// first index r in [lo, hi) with ends[r] > pos (ends non-decreasing); hi when none
__device__ __forceinline__ uint64_t upper_bound(const unsigned long long *ends, uint64_t lo, uint64_t hi, uint64_t pos)
{
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (ends[mid] > pos) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

template <int ES>
__global__ void __launch_bounds__(R_THREADS)
k_rle_expand(const unsigned long long *__restrict__ ends, uint64_t runs, const uint8_t *__restrict__ values,
             uint64_t n, uint8_t *__restrict__ out)
{
    __shared__ uint64_t s_lo, s_hi;
    const uint64_t t0 = (uint64_t)blockIdx.x * R_TILE;
    if (threadIdx.x == 0) {
        s_lo = upper_bound(ends, 0, runs, t0);
        const uint64_t last = t0 + R_TILE - 1 < n ? t0 + R_TILE - 1 : n - 1;
        uint64_t hi = upper_bound(ends, s_lo, runs, last);
        s_hi = hi < runs ? hi + 1 : runs;
    }
    __syncthreads();
    const uint64_t base = t0 + (uint64_t)threadIdx.x * R_PER;
    if (base >= n) return;
    uint64_t r = upper_bound(ends, s_lo, s_hi, base);
    uint64_t v[R_PER];
#pragma unroll
    for (int j = 0; j < R_PER; j++) {
        const uint64_t i = base + j;
        while (r < runs && ends[r] <= i) ++r;
        v[j] = (i < n && r < runs) ? ld_unaligned<ES>(values + r * ES) : 0;
    }
    if (base + R_PER <= n && (R_PER * ES) % 16 == 0) {
        constexpr int PER = 16 / ES;
#pragma unroll
        for (int c = 0; c < R_PER / PER; c++)
            reinterpret_cast<uint4 *>(out + (base + c * PER) * ES)[0] = make_chunk<ES>(v + c * PER);
    } else {
        for (int j = 0; j < R_PER; j++)
            if (base + j < n) st_elem<ES>(out, base + j, v[j]);
    }
}

}  // namespace

uint64_t rle_tiles(uint64_t n) { return (n + R_TILE - 1) / R_TILE; }

void launch_rle_encode(const uint8_t *in, uint64_t n, int es, Order o, uint8_t *values, int32_t *lengths,
                       uint32_t *starts, unsigned long long *runs, uint8_t *scratch, cudaStream_t s)
{
    if (n == 0) {
        GTSC_CUDA(cudaMemsetAsync(runs, 0, 8, s));
        return;
    }
    const uint64_t tiles = rle_tiles(n);
    GTSC_CUDA(cudaMemsetAsync(scratch, 0, lookback_zero_bytes(tiles), s));
    Lookback lb = lookback_at(scratch, tiles);
    switch (es) {
    case 1: k_rle_heads<1><<<(unsigned)tiles, R_THREADS, 0, s>>>(in, n, o, values, starts, runs, lb); break;
    case 2: k_rle_heads<2><<<(unsigned)tiles, R_THREADS, 0, s>>>(in, n, o, values, starts, runs, lb); break;
    case 4: k_rle_heads<4><<<(unsigned)tiles, R_THREADS, 0, s>>>(in, n, o, values, starts, runs, lb); break;
    default: k_rle_heads<8><<<(unsigned)tiles, R_THREADS, 0, s>>>(in, n, o, values, starts, runs, lb); break;
    }
    GTSC_CUDA(cudaGetLastError());
    uint64_t g = (n + 255) / 256;
    uint64_t cap = (uint64_t)sm_count() * 8;
    k_rle_lengths<<<(unsigned)(g < cap ? g : cap), 256, 0, s>>>(starts, runs, n, lengths);
    GTSC_CUDA(cudaGetLastError());
}

void launch_scan_i32(const uint8_t *in, uint64_t n, unsigned long long *out, uint8_t *scratch, cudaStream_t s)
{
    if (n == 0) return;
    const uint64_t tiles = rle_tiles(n);
    GTSC_CUDA(cudaMemsetAsync(scratch, 0, lookback_zero_bytes(tiles), s));
    Lookback lb = lookback_at(scratch, tiles);
    k_scan_i32<<<(unsigned)tiles, R_THREADS, 0, s>>>(in, n, out, lb);
    GTSC_CUDA(cudaGetLastError());
}

void launch_rle_expand(const unsigned long long *ends, uint64_t runs, const uint8_t *values, uint64_t n, int es,
                       uint8_t *out, cudaStream_t s)
{
    if (n == 0 || runs == 0) return;
    const uint64_t tiles = rle_tiles(n);
    switch (es) {
    case 1: k_rle_expand<1><<<(unsigned)tiles, R_THREADS, 0, s>>>(ends, runs, values, n, out); break;
    case 2: k_rle_expand<2><<<(unsigned)tiles, R_THREADS, 0, s>>>(ends, runs, values, n, out); break;
    case 4: k_rle_expand<4><<<(unsigned)tiles, R_THREADS, 0, s>>>(ends, runs, values, n, out); break;
    default: k_rle_expand<8><<<(unsigned)tiles, R_THREADS, 0, s>>>(ends, runs, values, n, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
