// delta_scale.cu -- delta and scale encodings (wrapping integer arithmetic on element bits).
//
// DeltaEncoding (compression/delta/delta_encoding.cu:19-102): out[i] = x[i+1] - x[i]; decode is an
// inclusive scan plus the first value.  The reference runs an elementwise kernel then a Thrust
// scan plus a second "add first" pass; here decode is ONE pass: each tile's prefix comes from a
// decoupled look-back (scan.cuh) and the first value is added as the result is stored.
// ScaleEncoding (compression/scale/scale_encoding.cu:21-108): out[i] = x[i] - min, decode adds it
// back; the kernels read `min` from the metadata buffer on the device.
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int EW_THREADS = 256;

template <int ES>
__device__ __forceinline__ uint64_t wrap(uint64_t v)
{
    return ES == 8 ? v : (v & ((1ull << (8 * ES)) - 1));
}

// ---------------------------------------------------------------- delta encode
template <int ES>
__global__ void __launch_bounds__(EW_THREADS)
k_delta_encode(const uint8_t *__restrict__ in, uint64_t n, uint8_t *__restrict__ out)
{
    constexpr int PER = 16 / ES;
    const uint64_t m = n - 1;  // outputs
    const uint64_t chunks = (m + PER - 1) / PER;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < chunks; c += stride) {
        const uint64_t i0 = c * PER;
        uint64_t v[PER + 1], d[PER];
        if (i0 + PER < n) {
            uint4 ch = ld_chunk(in + 16 * c);
#pragma unroll
            for (int j = 0; j < PER; j++) v[j] = chunk_elem<ES>(ch, j);
            v[PER] = ld_elem<ES>(in, i0 + PER);
#pragma unroll
            for (int j = 0; j < PER; j++) d[j] = wrap<ES>(v[j + 1] - v[j]);
            if (i0 + PER <= m) {
                reinterpret_cast<uint4 *>(out)[c] = make_chunk<ES>(d);
                continue;
            }
        } else {
            for (int j = 0; j <= PER; j++) v[j] = i0 + j < n ? ld_elem<ES>(in, i0 + j) : 0;
            for (int j = 0; j < PER; j++) d[j] = wrap<ES>(v[j + 1] - v[j]);
        }
        for (int j = 0; j < PER; j++)
            if (i0 + j < m) st_elem<ES>(out, i0 + j, d[j]);
    }
}

// ---------------------------------------------------------------- delta decode (one pass)
constexpr int DD_THREADS = 256;
constexpr int DD_PER = 8;  // elements per thread
constexpr int DD_TILE = DD_THREADS * DD_PER;

template <int ES>
__global__ void __launch_bounds__(DD_THREADS)
k_delta_decode(const uint8_t *__restrict__ d, uint64_t n, const uint8_t *__restrict__ first_p,
               uint8_t *__restrict__ out, Lookback lb)
{
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t s_tile;
    const uint64_t m = n - 1;  // deltas
    if (threadIdx.x == 0) s_tile = claim_tile(lb);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * DD_TILE + (uint64_t)threadIdx.x * DD_PER;
    uint64_t v[DD_PER];
#pragma unroll
    for (int j = 0; j < DD_PER; j++) v[j] = base + j < m ? ld_elem<ES>(d, base + j) : 0;
    unsigned long long local = 0;
#pragma unroll
    for (int j = 0; j < DD_PER; j++) local += v[j];
    unsigned long long total;
    unsigned long long excl = block_exclusive_scan<DD_THREADS>(local, ws, total);
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    unsigned long long acc = ld_unaligned<ES>(first_p) + s_prefix + excl;
    uint64_t o[DD_PER];
#pragma unroll
    for (int j = 0; j < DD_PER; j++) {
        o[j] = wrap<ES>(acc);
        acc += v[j];
    }
    if (base + DD_PER <= n && (DD_PER * ES) % 16 == 0) {
        constexpr int PER = 16 / ES;
#pragma unroll
        for (int c = 0; c < DD_PER / PER; c++)
            reinterpret_cast<uint4 *>(out + (base + c * PER) * ES)[0] = make_chunk<ES>(o + c * PER);
    } else {
        for (int j = 0; j < DD_PER; j++)
            if (base + j < n) st_elem<ES>(out, base + j, o[j]);
    }
}

// ---------------------------------------------------------------- scale
template <int ES, bool ENC>
__global__ void __launch_bounds__(EW_THREADS)
k_scale(const uint8_t *__restrict__ in, uint64_t n, const uint8_t *__restrict__ min_p, uint8_t *__restrict__ out)
{
    constexpr int PER = 16 / ES;
    const uint64_t mn = ld_unaligned<ES>(min_p);
    const uint64_t chunks = (n + PER - 1) / PER;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < chunks; c += stride) {
        const uint64_t i0 = c * PER;
        uint64_t v[PER];
        if (i0 + PER <= n) {
            uint4 ch = ld_chunk(in + 16 * c);
#pragma unroll
            for (int j = 0; j < PER; j++) v[j] = wrap<ES>(ENC ? chunk_elem<ES>(ch, j) - mn : chunk_elem<ES>(ch, j) + mn);
            reinterpret_cast<uint4 *>(out)[c] = make_chunk<ES>(v);
        } else {
            for (int j = 0; j < PER; j++)
                if (i0 + j < n) {
                    uint64_t x = ld_elem<ES>(in, i0 + j);
                    st_elem<ES>(out, i0 + j, ENC ? x - mn : x + mn);
                }
        }
    }
}

unsigned ew_grid(uint64_t items)
{
    uint64_t b = (items + EW_THREADS - 1) / EW_THREADS;
    uint64_t cap = (uint64_t)sm_count() * 8;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

}  // namespace

void launch_delta_encode(const uint8_t *in, uint64_t n, int es, uint8_t *out, cudaStream_t s)
{
    if (n < 2) return;
    const uint64_t chunks = ((n - 1) * es + 15) / 16;
    const unsigned g = ew_grid(chunks);
    switch (es) {
    case 1: k_delta_encode<1><<<g, EW_THREADS, 0, s>>>(in, n, out); break;
    case 2: k_delta_encode<2><<<g, EW_THREADS, 0, s>>>(in, n, out); break;
    case 4: k_delta_encode<4><<<g, EW_THREADS, 0, s>>>(in, n, out); break;
    default: k_delta_encode<8><<<g, EW_THREADS, 0, s>>>(in, n, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

uint64_t delta_decode_tiles(uint64_t n) { return (n + DD_TILE - 1) / DD_TILE; }

void launch_delta_decode(const uint8_t *d, uint64_t n, const uint8_t *first, uint8_t *out,
                         uint8_t *scratch, int es, cudaStream_t s)
{
    if (n == 0) return;
    const uint64_t tiles = delta_decode_tiles(n);
    GTSC_CUDA(cudaMemsetAsync(scratch, 0, lookback_zero_bytes(tiles), s));
    Lookback lb = lookback_at(scratch, tiles);
    switch (es) {
    case 1: k_delta_decode<1><<<(unsigned)tiles, DD_THREADS, 0, s>>>(d, n, first, out, lb); break;
    case 2: k_delta_decode<2><<<(unsigned)tiles, DD_THREADS, 0, s>>>(d, n, first, out, lb); break;
    case 4: k_delta_decode<4><<<(unsigned)tiles, DD_THREADS, 0, s>>>(d, n, first, out, lb); break;
    default: k_delta_decode<8><<<(unsigned)tiles, DD_THREADS, 0, s>>>(d, n, first, out, lb); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_scale(const uint8_t *in, uint64_t n, int es, const uint8_t *min_p, uint8_t *out, bool encode,
                  cudaStream_t s)
{
    if (n == 0) return;
    const unsigned g = ew_grid((n * es + 15) / 16);
#define GTSC_SCALE_CASE(E)                                                                   \
    if (encode) k_scale<E, true><<<g, EW_THREADS, 0, s>>>(in, n, min_p, out);                \
    else k_scale<E, false><<<g, EW_THREADS, 0, s>>>(in, n, min_p, out);
    switch (es) {
    case 1: GTSC_SCALE_CASE(1) break;
    case 2: GTSC_SCALE_CASE(2) break;
    case 4: GTSC_SCALE_CASE(4) break;
    default: GTSC_SCALE_CASE(8) break;
    }
#undef GTSC_SCALE_CASE
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
