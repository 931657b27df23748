// afl.cu -- AFL/FL fixed-width bit packing for sm_100a.
//
// Layout (what run_afl_compress_gpu<T,1> of compression/afl/afl_gpu.cu:67-73,124-163 produces for
// the AflEncoding, afl_encoding.cu:45): value i occupies bits [i*b, i*b+b) of one little-endian,
// LSB-first bitstream, padded with zero bits to a whole T word.  The reference gives each thread
// 32 consecutive values (8-thread blocks, 4-byte strided accesses); here the roles are swapped:
//
//  pack   -- a block stages a tile of 2048 values in shared memory with 16-byte coalesced loads,
//            then every thread builds whole 32-bit output words by gathering the <= 32/b + 1
//            values that cover each word (shift / OR in a 64-bit register) and stores them
//            coalesced.  Reads n*es bytes once, writes the stream once.
//  unpack -- every thread extracts 4 consecutive values with funnel shifts from the (L1-cached)
//            32-bit words covering them and writes them with one vector store.
#include "kernels.hpp"
#include "vec.cuh"

#include <type_traits>

namespace gtsc {

namespace {

constexpr int AFL_THREADS = 256;
constexpr int AFL_TILE = 2048;  // values per tile; multiple of 32 so tiles start on word edges

template <int ES, bool WIDE>
__global__ void __launch_bounds__(AFL_THREADS)
k_afl_pack(const uint8_t *__restrict__ in, uint64_t n, int b, uint8_t *__restrict__ out,
           uint64_t out_bytes)
{
    using V = typename std::conditional<WIDE, unsigned long long, uint32_t>::type;
    __shared__ V sv[AFL_TILE + 4];
    const uint64_t vmask = b >= 64 ? ~0ull : ((1ull << b) - 1);
    const uint64_t total_words = (out_bytes + 3) / 4;
    const uint64_t ntiles = (n + AFL_TILE - 1) / AFL_TILE;
    const int tid = threadIdx.x;

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t t0 = tile * AFL_TILE;
        const uint64_t cnt = n - t0 < (uint64_t)AFL_TILE ? n - t0 : (uint64_t)AFL_TILE;
        const uint8_t *src = in + t0 * ES;
        if (cnt == (uint64_t)AFL_TILE) {
            constexpr int PER = 16 / ES;
            for (int c = tid; c < AFL_TILE / PER; c += AFL_THREADS) {
                uint4 v = ld_chunk(src + 16 * c);
#pragma unroll
                for (int j = 0; j < PER; j++) sv[c * PER + j] = (V)(chunk_elem<ES>(v, j) & vmask);
            }
        } else {
            for (int i = tid; i < AFL_TILE; i += AFL_THREADS)
                sv[i] = (uint64_t)i < cnt ? (V)(ld_elem<ES>(src, i) & vmask) : (V)0;
        }
        if (tid < 4) sv[AFL_TILE + tid] = 0;
        __syncthreads();

        const uint64_t w0 = t0 * (uint64_t)b / 32;
        uint64_t w_end = (t0 + AFL_TILE) * (uint64_t)b / 32;
        if (w_end > total_words) w_end = total_words;
        for (uint64_t w = w0 + tid; w < w_end; w += AFL_THREADS) {
            const uint32_t p = (uint32_t)(w - w0) * 32u;
            uint32_t a = p / (uint32_t)b;
            const uint32_t s = p - a * (uint32_t)b;
            uint32_t word;
            if (!WIDE) {
                uint64_t acc = (uint64_t)sv[a] >> s;
                int filled = b - (int)s;
                ++a;
                while (filled < 32) {
                    acc |= (uint64_t)sv[a] << filled;
                    filled += b;
                    ++a;
                }
                word = (uint32_t)acc;
            } else {
                uint64_t acc = (uint64_t)sv[a] >> s;
                const int filled = b - (int)s;
                if (filled < 32) acc |= (uint64_t)sv[a + 1] << filled;
                word = (uint32_t)acc;
            }
            if (4 * w + 4 <= out_bytes) {
                reinterpret_cast<uint32_t *>(out)[w] = word;
            } else {
                for (int k = 0; k < 4; k++)
                    if (4 * w + k < out_bytes) out[4 * w + k] = (uint8_t)(word >> (8 * k));
            }
        }
        __syncthreads();
    }
}

template <int ES>
__global__ void __launch_bounds__(256)
k_afl_unpack(StreamReader rd, uint32_t off_bits, uint64_t n, int b, uint8_t *__restrict__ out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = b >= 64 ? ~0ull : ((1ull << b) - 1);
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q * 4 < n; q += stride) {
        const uint64_t i0 = q * 4;
        uint64_t v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint64_t i = i0 + j;
            v[j] = 0;
            if (i < n) {
                const uint64_t p = off_bits + i * (uint64_t)b;
                const uint64_t w = p >> 5;
                const uint32_t s = (uint32_t)(p & 31);
                if (b <= 32) {
                    const uint32_t lo = rd.word(w);
                    const uint32_t hi = (s + b > 32) ? rd.word(w + 1) : 0u;
                    v[j] = __funnelshift_r(lo, hi, s) & mask;
                } else {
                    const uint64_t q0 = (uint64_t)rd.word(w) | ((uint64_t)rd.word(w + 1) << 32);
                    uint64_t x = q0 >> s;
                    if (s + b > 64) x |= (uint64_t)rd.word(w + 2) << (64 - s);
                    v[j] = x & mask;
                }
            }
        }
        if (i0 + 3 < n) {
            if (ES == 4) {
                reinterpret_cast<uint4 *>(out)[q] = make_uint4((uint32_t)v[0], (uint32_t)v[1], (uint32_t)v[2], (uint32_t)v[3]);
            } else if (ES == 8) {
                uint4 *o = reinterpret_cast<uint4 *>(out) + 2 * q;
                o[0] = make_uint4((uint32_t)v[0], (uint32_t)(v[0] >> 32), (uint32_t)v[1], (uint32_t)(v[1] >> 32));
                o[1] = make_uint4((uint32_t)v[2], (uint32_t)(v[2] >> 32), (uint32_t)v[3], (uint32_t)(v[3] >> 32));
            } else if (ES == 2) {
                reinterpret_cast<uint2 *>(out)[q] =
                    make_uint2((uint32_t)v[0] | ((uint32_t)v[1] << 16), (uint32_t)v[2] | ((uint32_t)v[3] << 16));
            } else {
                reinterpret_cast<uint32_t *>(out)[q] =
                    (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
            }
        } else {
            for (int j = 0; j < 4; j++)
                if (i0 + j < n) st_elem<ES>(out, i0 + j, v[j]);
        }
    }
}

template <int ES>
void pack_es(const uint8_t *in, uint64_t n, int b, uint8_t *out, uint64_t out_bytes, cudaStream_t s)
{
    uint64_t tiles = (n + AFL_TILE - 1) / AFL_TILE;
    uint64_t cap = (uint64_t)sm_count() * 8;
    unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    if (b > 32) k_afl_pack<ES, true><<<grid, AFL_THREADS, 0, s>>>(in, n, b, out, out_bytes);
    else k_afl_pack<ES, false><<<grid, AFL_THREADS, 0, s>>>(in, n, b, out, out_bytes);
}

}  // namespace

void launch_afl_pack(const uint8_t *in, uint64_t n, int es, int b, uint8_t *out, uint64_t out_bytes,
                     cudaStream_t s)
{
    if (n == 0 || out_bytes == 0) return;
    if (((uintptr_t)in & 15) || ((uintptr_t)out & 3)) fail(GTSC_ERR_ARG, "afl pack: misaligned buffer");
    if (b < 1 || b > 8 * es) fail(GTSC_ERR_ARG, "afl pack: bad bit width");
    switch (es) {
    case 1: pack_es<1>(in, n, b, out, out_bytes, s); break;
    case 2: pack_es<2>(in, n, b, out, out_bytes, s); break;
    case 4: pack_es<4>(in, n, b, out, out_bytes, s); break;
    default: pack_es<8>(in, n, b, out, out_bytes, s); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

void launch_afl_unpack(const uint8_t *stream, uint64_t stream_bytes, uint64_t n, int es, int b,
                       uint8_t *out, cudaStream_t s)
{
    if (n == 0) return;
    if (b < 1 || b > 8 * es) fail(GTSC_ERR_FORMAT, "afl unpack: bad bit width");
    if ((uintptr_t)out & 15) fail(GTSC_ERR_ARG, "afl unpack: misaligned output");
    const uintptr_t mis = (uintptr_t)stream & 3;
    StreamReader rd{reinterpret_cast<const uint32_t *>(stream - mis), stream_bytes + mis};
    const uint32_t off_bits = (uint32_t)(8 * mis);
    uint64_t quads = (n + 3) / 4;
    uint64_t blocks = (quads + 255) / 256;
    uint64_t cap = (uint64_t)sm_count() * 8;
    unsigned grid = (unsigned)(blocks < cap ? blocks : cap);
    switch (es) {
    case 1: k_afl_unpack<1><<<grid, 256, 0, s>>>(rd, off_bits, n, b, out); break;
    case 2: k_afl_unpack<2><<<grid, 256, 0, s>>>(rd, off_bits, n, b, out); break;
    case 4: k_afl_unpack<4><<<grid, 256, 0, s>>>(rd, off_bits, n, b, out); break;
    default: k_afl_unpack<8><<<grid, 256, 0, s>>>(rd, off_bits, n, b, out); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
