// afl32.cu -- the aligned AFL layout (CWARP_SIZE = 32, compression/afl/afl_gpu.cu:253-269) and
// random-access decoding of either layout (afl_decompress_base_value_gpu, afl_gpu.cu:113-121 and
// 197-222).
//
// Aligned layout, W = bits of an element: values come in blocks of 32*W; value j of lane l of block
// B is element B*32W + 32j + l, and lane l packs its values (LSB first) into the words
// B*32b + 32k + l, k = 0..b-1.  A lane that runs out of elements inside the block's last row
// (its next element index lies in [n, n + 32)) also stores its last, partial word, whatever the
// word count; the total is ceil(n / 32W) * 32b words.
//
// FL layout (omega 1): value i at bits [i*b, i*b + b) of the word stream (the one AflEncoding
// uses; packed by afl.cu).
#include "kernels.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

// the packed word type of an element width: 32-bit arithmetic for elements of up to 4 bytes
template <int ES> struct WordOf { using T = uint32_t; };
template <> struct WordOf<8> { using T = unsigned long long; };

template <typename T>
__device__ __forceinline__ T low_mask(int bits)
{
    return bits >= (int)(8 * sizeof(T)) ? ~T(0) : ((T(1) << bits) - 1);
}

// one thread = one lane of one block of 32*W elements
template <int ES>
__global__ void __launch_bounds__(256) k_afl32_pack(const uint8_t *__restrict__ in, uint64_t n, int b,
                                                    uint8_t *__restrict__ out, uint64_t words)
{
    using T = typename WordOf<ES>::T;
    constexpr int W = 8 * ES;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t blk = t >> 5, lane = t & 31;
    const uint64_t first = blk * 32ull * W + lane;
    if (blk * 32ull * W >= n) return;
    const T vmask = low_mask<T>(b), wmask = low_mask<T>(W);
    T acc = 0;
    uint64_t wpos = blk * 32ull * b + lane;
    int fill = 0;
    if ((blk + 1) * 32ull * W <= n) {  // a whole block: every load first, then the packing
        T v[W];
#pragma unroll
        for (int j = 0; j < W; j++) v[j] = (T)ld_elem<ES>(in, first + 32ull * j) & vmask;
#pragma unroll
        for (int j = 0; j < W; j++) {
            acc |= (v[j] << fill) & wmask;
            if (fill >= W - b) {  // the word is full
                st_elem<ES>(out, wpos, acc);
                wpos += 32;
                const int used = W - fill;
                fill = b - used;
                acc = used >= W ? T(0) : (v[j] >> used) & low_mask<T>(fill);
            } else {
                fill += b;
            }
        }
        return;  // the last word of a whole block ends exactly at bit W*b
    }
    uint64_t idx = first;
    for (int j = 0; j < W && idx < n; j++, idx += 32) {
        const T x = (T)ld_elem<ES>(in, idx) & vmask;
        acc |= (x << fill) & wmask;
        if (fill >= W - b) {
            if (wpos < words) st_elem<ES>(out, wpos, acc);
            wpos += 32;
            const int used = W - fill;
            fill = b - used;
            acc = used >= W ? T(0) : (x >> used) & low_mask<T>(fill);
        } else {
            fill += b;
        }
    }
    if (idx >= n && idx < n + 32 && wpos < words) st_elem<ES>(out, wpos, acc);
}

template <int ES>
__global__ void __launch_bounds__(256) k_afl32_unpack(const uint8_t *__restrict__ comp, uint64_t words, int b,
                                                      uint64_t n, uint8_t *__restrict__ out)
{
    using T = typename WordOf<ES>::T;
    constexpr int W = 8 * ES;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t blk = t >> 5, lane = t & 31;
    uint64_t idx = blk * 32ull * W + lane;
    if (blk * 32ull * W >= n) return;
    const T vmask = low_mask<T>(b);
    uint64_t wpos = blk * 32ull * b + lane;
    T cur = wpos < words ? (T)ld_elem<ES>(comp, wpos) : T(0);
    int pos = 0;
    for (int j = 0; j < W && idx < n; j++, idx += 32) {
        T v;
        if (pos > W - b) {  // the value continues in the lane's next word
            const int have = W - pos;
            v = (cur >> pos) & low_mask<T>(have);
            wpos += 32;
            cur = wpos < words ? (T)ld_elem<ES>(comp, wpos) : T(0);
            pos = b - have;
            v |= (cur & low_mask<T>(pos)) << have;
        } else {
            v = (cur >> pos) & vmask;
            pos += b;
            if (pos == W && j + 1 < W) {  // the next value starts a new word
                wpos += 32;
                cur = wpos < words ? (T)ld_elem<ES>(comp, wpos) : T(0);
                pos = 0;
            }
        }
        st_elem<ES>(out, idx, v);
    }
}

// element i of a packed stream, OMEGA = 1 (FL) or 32 (aligned); words past the stream read 0
template <int ES, int OMEGA, typename I>
__device__ __forceinline__ uint64_t afl_value(const uint8_t *comp, I words, int b, I i)
{
    using T = typename WordOf<ES>::T;
    constexpr int W = 8 * ES;
    constexpr I per = (I)OMEGA * W;
    const I blk = i / per, in_blk = i % per;
    const uint32_t lane = (uint32_t)(in_blk % OMEGA), row = (uint32_t)(in_blk / OMEGA);
    const uint32_t rb = row * (uint32_t)b;
    const I word = blk * (I)(OMEGA * b) + lane + (I)(rb / W) * OMEGA;
    const int bit = (int)(rb % W);
    const int first = bit <= W - b ? b : W - bit;
    T v = word < words ? ((T)ld_elem<ES>(comp, word) >> bit) & low_mask<T>(first) : T(0);
    if (first < b) {
        const I w2 = word + OMEGA;
        const T hi = w2 < words ? (T)ld_elem<ES>(comp, w2) & low_mask<T>(b - first) : T(0);
        v |= hi << first;
    }
    return v;
}

template <int ES, int OMEGA>
__global__ void __launch_bounds__(256) k_afl_values(const uint8_t *__restrict__ comp, uint64_t words, int b,
                                                    const uint64_t *__restrict__ idx, uint64_t n,
                                                    uint8_t *__restrict__ out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t i = idx ? __ldg(idx + t) : t;
    // 32-bit index arithmetic while it cannot wrap (the words read lie below i + 2 * OMEGA)
    const uint64_t v = i < 0xffffff00ull && words < 0xffffff00ull
                           ? afl_value<ES, OMEGA, uint32_t>(comp, (uint32_t)words, b, (uint32_t)i)
                           : afl_value<ES, OMEGA, uint64_t>(comp, words, b, i);
    st_elem<ES>(out, t, v);
}

// Every element of an aligned (omega 32) stream, 16 bytes of output a thread: its 16 / ES elements
// are consecutive lanes of one row of one block, so their words are consecutive too -- one 16-byte
// load of the row's words (and one of the next row's when the values cross into it), shifts, one
// 16-byte store.  Rows whose words reach past the stream, and a ragged end, take the element path.
template <int ES>
__global__ void __launch_bounds__(256) k_afl32_values_all(const uint8_t *__restrict__ comp, uint64_t words, int b,
                                                          uint64_t n, uint8_t *__restrict__ out)
{
    using T = typename WordOf<ES>::T;
    constexpr int W = 8 * ES, V = 16 / ES;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t e0 = t * V;
    if (e0 >= n) return;
    const uint64_t per = 32ull * W;
    const uint64_t blk = e0 / per, in_blk = e0 % per;
    const uint32_t lane0 = (uint32_t)(in_blk % 32), row = (uint32_t)(in_blk / 32);
    const uint32_t rb = row * (uint32_t)b;
    const uint64_t word = blk * 32ull * b + lane0 + (uint64_t)(rb / W) * 32;
    const int bit = (int)(rb % W);
    const bool cross = bit > W - b;
    if (e0 + V > n || word + V + (cross ? 32 : 0) > words) {
        for (int j = 0; j < V && e0 + j < n; j++)
            st_elem<ES>(out, e0 + j, afl_value<ES, 32, uint64_t>(comp, words, b, e0 + j));
        return;
    }
    const uint4 lo = ld_chunk(comp + word * ES);
    uint4 hi = make_uint4(0, 0, 0, 0);
    if (cross) hi = ld_chunk(comp + (word + 32) * ES);
    const T mask = low_mask<T>(b);
    uint64_t v[V];
#pragma unroll
    for (int j = 0; j < V; j++) {
        const T a = (T)chunk_elem<ES>(lo, j);
        T x = a >> bit;
        if (cross) x |= (T)chunk_elem<ES>(hi, j) << (W - bit);
        v[j] = x & mask;
    }
    reinterpret_cast<uint4 *>(out + e0 * ES)[0] = make_chunk<ES>(v);
}

template <int ES>
void values_es(const uint8_t *comp, uint64_t words, int b, int omega, const uint64_t *idx, uint64_t n, uint8_t *out,
               cudaStream_t s)
{
    if (omega == 32 && !idx && ((uintptr_t)comp & 15) == 0 && ((uintptr_t)out & 15) == 0) {
        const uint64_t threads = (n + 16 / ES - 1) / (16 / ES);
        k_afl32_values_all<ES><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(comp, words, b, n, out);
        return;
    }
    const unsigned g = (unsigned)((n + 255) / 256);
    if (omega == 32) k_afl_values<ES, 32><<<g, 256, 0, s>>>(comp, words, b, idx, n, out);
    else k_afl_values<ES, 1><<<g, 256, 0, s>>>(comp, words, b, idx, n, out);
}

}  // namespace

uint64_t afl32_words(uint64_t n, int b, int es)
{
    const uint64_t per = 32ull * 8 * es;
    return (n + per - 1) / per * 32ull * b;
}

void launch_afl32_pack(const uint8_t *in, uint64_t n, int es, int b, uint8_t *out, uint64_t words, cudaStream_t s)
{
    if (!n) return;
    const uint64_t threads = (n + 32ull * 8 * es - 1) / (32ull * 8 * es) * 32;
    const unsigned g = (unsigned)((threads + 255) / 256);
    switch (es) {
    case 1: k_afl32_pack<1><<<g, 256, 0, s>>>(in, n, b, out, words); break;
    case 2: k_afl32_pack<2><<<g, 256, 0, s>>>(in, n, b, out, words); break;
    case 4: k_afl32_pack<4><<<g, 256, 0, s>>>(in, n, b, out, words); break;
    default: k_afl32_pack<8><<<g, 256, 0, s>>>(in, n, b, out, words); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_afl32_unpack(const uint8_t *comp, uint64_t words, uint64_t n, int es, int b, uint8_t *out, cudaStream_t s)
{
    if (!n) return;
    const uint64_t threads = (n + 32ull * 8 * es - 1) / (32ull * 8 * es) * 32;
    const unsigned g = (unsigned)((threads + 255) / 256);
    switch (es) {
    case 1: k_afl32_unpack<1><<<g, 256, 0, s>>>(comp, words, b, n, out); break;
    case 2: k_afl32_unpack<2><<<g, 256, 0, s>>>(comp, words, b, n, out); break;
    case 4: k_afl32_unpack<4><<<g, 256, 0, s>>>(comp, words, b, n, out); break;
    default: k_afl32_unpack<8><<<g, 256, 0, s>>>(comp, words, b, n, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_afl_values(const uint8_t *comp, uint64_t words, int es, int b, int omega, const uint64_t *idx,
                       uint64_t n, uint8_t *out, cudaStream_t s)
{
    if (!n) return;
    switch (es) {
    case 1: values_es<1>(comp, words, b, omega, idx, n, out, s); break;
    case 2: values_es<2>(comp, words, b, omega, idx, n, out, s); break;
    case 4: values_es<4>(comp, words, b, omega, idx, n, out, s); break;
    default: values_es<8>(comp, words, b, omega, idx, n, out, s); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
