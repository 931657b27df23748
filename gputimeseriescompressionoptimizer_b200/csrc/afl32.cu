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

template <int ES>
__device__ __forceinline__ uint64_t afl_mask(int bits)
{
    return bits >= 64 ? ~0ull : ((1ull << bits) - 1);
}

template <int ES>
__device__ __forceinline__ void st_word(uint8_t *p, uint64_t i, uint64_t v)
{
    st_elem<ES>(p, i, v);
}

// one thread = one lane of one block
template <int ES>
__global__ void k_afl32_pack(const uint8_t *__restrict__ in, uint64_t n, int b, uint8_t *__restrict__ out,
                             uint64_t words)
{
    constexpr int W = 8 * ES;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t blk = t / 32, lane = t % 32;
    const uint64_t first = blk * 32ull * W + lane;
    if (blk * 32ull * W >= n) return;
    const uint64_t vmask = afl_mask<ES>(b), wmask = afl_mask<ES>(W);
    uint64_t acc = 0, idx = first, wpos = blk * 32ull * b + lane;
    int fill = 0;
    for (int j = 0; j < W && idx < n; j++, idx += 32) {
        const uint64_t x = ld_elem<ES>(in, idx) & vmask;
        acc |= (x << fill) & wmask;
        if (fill >= W - b) {  // the word is full
            if (wpos < words) st_word<ES>(out, wpos, acc);
            wpos += 32;
            const int used = W - fill;  // bits of x in the word just written
            fill = b - used;
            acc = used >= 64 ? 0 : (x >> used) & afl_mask<ES>(fill);
        } else {
            fill += b;
        }
    }
    if (idx >= n && idx < n + 32 && wpos < words) st_word<ES>(out, wpos, acc);
}

template <int ES>
__global__ void k_afl32_unpack(const uint8_t *__restrict__ comp, uint64_t words, int b, uint64_t n,
                               uint8_t *__restrict__ out)
{
    constexpr int W = 8 * ES;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t blk = t / 32, lane = t % 32;
    uint64_t idx = blk * 32ull * W + lane;
    if (blk * 32ull * W >= n) return;
    const uint64_t vmask = afl_mask<ES>(b);
    uint64_t wpos = blk * 32ull * b + lane;
    uint64_t cur = wpos < words ? ld_elem<ES>(comp, wpos) : 0;
    int pos = 0;
    for (int j = 0; j < W && idx < n; j++, idx += 32) {
        uint64_t v;
        if (pos > W - b) {  // the value continues in the lane's next word
            const int have = W - pos;
            v = (cur >> pos) & afl_mask<ES>(have);
            wpos += 32;
            cur = wpos < words ? ld_elem<ES>(comp, wpos) : 0;
            pos = b - have;
            v |= (cur & afl_mask<ES>(pos)) << have;
        } else {
            v = (cur >> pos) & vmask;
            pos += b;
            if (pos == W && j + 1 < W) {  // the next value starts a new word
                wpos += 32;
                cur = wpos < words ? ld_elem<ES>(comp, wpos) : 0;
                pos = 0;
            }
        }
        st_elem<ES>(out, idx, v);
    }
}

// element i of a packed stream; omega = 1 (FL) or 32 (aligned)
template <int ES>
__device__ __forceinline__ uint64_t afl_value(const uint8_t *comp, uint64_t words, int b, int omega, uint64_t i)
{
    constexpr int W = 8 * ES;
    const uint64_t per = (uint64_t)omega * W;
    const uint64_t blk = i / per, in_blk = i % per;
    const uint64_t lane = in_blk % omega, row = in_blk / omega;
    const uint64_t word = blk * (uint64_t)omega * b + lane + (row * b / W) * omega;
    const int bit = (int)(row * b % W);
    const int first = bit <= W - b ? b : W - bit;
    uint64_t v = word < words ? (ld_elem<ES>(comp, word) >> bit) & afl_mask<ES>(first) : 0;
    if (first < b) {
        const uint64_t w2 = word + omega;
        const uint64_t hi = w2 < words ? ld_elem<ES>(comp, w2) & afl_mask<ES>(b - first) : 0;
        v |= hi << first;
    }
    return v;
}

template <int ES>
__global__ void k_afl_values(const uint8_t *__restrict__ comp, uint64_t words, int b, int omega,
                             const uint64_t *__restrict__ idx, uint64_t n, uint8_t *__restrict__ out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t i = idx ? idx[t] : t;
    st_elem<ES>(out, t, afl_value<ES>(comp, words, b, omega, i));
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
    const unsigned g = (unsigned)((n + 255) / 256);
    switch (es) {
    case 1: k_afl_values<1><<<g, 256, 0, s>>>(comp, words, b, omega, idx, n, out); break;
    case 2: k_afl_values<2><<<g, 256, 0, s>>>(comp, words, b, omega, idx, n, out); break;
    case 4: k_afl_values<4><<<g, 256, 0, s>>>(comp, words, b, omega, idx, n, out); break;
    default: k_afl_values<8><<<g, 256, 0, s>>>(comp, words, b, omega, idx, n, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
