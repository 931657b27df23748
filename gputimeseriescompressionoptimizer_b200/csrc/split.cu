// split.cu -- stencil split / merge used by patch, const and dict, each in ONE pass.
//
// The reference builds these from several passes: a predicate kernel writing one int per element
// (Stencil::Create, util/stencil/stencil.cu:98-120), two Thrust exclusive scans and a scatter
// (Splitter::Split, util/splitter/splitter.cu:66-100), a pack kernel for the stencil bits
// (stencil.cu:14-68) and, for dict, UniqueEncoding's code kernel (unique_encoding.cu:48-131).
// Here a thread owns 8 consecutive elements -- exactly one stencil byte -- and a 2048-element tile
// gets its output offsets from a block scan plus a decoupled look-back (scan.cuh), so one read of
// the column produces the packed stencil, the two ordered streams and the dict codes.
#include "kernels.hpp"
#include "scan.cuh"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int SP_THREADS = 256;
constexpr int SP_PER = 8;
constexpr int SP_TILE = SP_THREADS * SP_PER;

// identity used for dictionary matches: equal bits, and never NaN (see or_common.h same_val)
__device__ __forceinline__ bool same_val(uint64_t a, uint64_t b, Order o) { return a == b && !is_nan_bits(a, o); }

template <int ES>
__device__ __forceinline__ void load8(const uint8_t *in, uint64_t base, uint64_t n, uint64_t *v)
{
    if (base + SP_PER <= n && ((uintptr_t)(in + base * ES) & 15) == 0 && (SP_PER * ES) % 16 == 0) {
        constexpr int PER = 16 / ES;
#pragma unroll
        for (int c = 0; c < SP_PER / PER; c++) {
            uint4 ch = ld_chunk(in + (base + c * PER) * ES);
#pragma unroll
            for (int j = 0; j < PER; j++) v[c * PER + j] = chunk_elem<ES>(ch, j);
        }
    } else {
#pragma unroll
        for (int j = 0; j < SP_PER; j++) v[j] = base + j < n ? ld_elem<ES>(in, base + j) : 0;
    }
}

template <int ES>
__device__ __forceinline__ void store8(uint8_t *out, uint64_t base, uint64_t n, const uint64_t *v)
{
    if (base + SP_PER <= n && (SP_PER * ES) % 16 == 0) {
        constexpr int PER = 16 / ES;
#pragma unroll
        for (int c = 0; c < SP_PER / PER; c++)
            reinterpret_cast<uint4 *>(out + (base + c * PER) * ES)[0] = make_chunk<ES>(v + c * PER);
    } else {
        for (int j = 0; j < SP_PER; j++)
            if (base + j < n) st_elem<ES>(out, base + j, v[j]);
    }
}

// ------------------------------------------------------------------------------ split
template <int ES, int MODE>
__global__ void __launch_bounds__(SP_THREADS)
k_split(const uint8_t *__restrict__ in, uint64_t n, SplitArgs a, Lookback lb)
{
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = claim_tile(lb);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * SP_TILE + (uint64_t)threadIdx.x * SP_PER;
    uint64_t v[SP_PER];
    load8<ES>(in, base, n, v);
    uint64_t top[4] = {0, 0, 0, 0};
    if (MODE != SPLIT_LOWER) {
#pragma unroll
        for (int k = 0; k < (MODE == SPLIT_DICT ? 4 : 1); k++) top[k] = ld_unaligned<ES>(a.top + k * ES);
    }

    // predicate and (dict) code of each element
    uint32_t bits = 0, codes = 0;
#pragma unroll
    for (int j = 0; j < SP_PER; j++) {
        bool f = false;
        uint32_t code = 0;
        if (MODE == SPLIT_LOWER) {
            f = a.outside ? !(lt_native(a.hi, v[j], ES, a.order) || lt_native(v[j], a.lo, ES, a.order))
                          : lt_native(v[j], a.thr, ES, a.order);
        } else if (MODE == SPLIT_NOT_CONST) {
            f = !same_val(v[j], top[0], a.order);
        } else {  // SPLIT_DICT
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (same_val(v[j], top[k], a.order)) { f = true; code |= (uint32_t)k; }
        }
        bits |= (uint32_t)f << j;
        codes |= code << (2 * j);
    }
    // stencil byte: bits past n repeat the last element's bit (stencil.cu:27)
    if (base < n) {
        const uint64_t valid = n - base;
        if (valid < SP_PER) {
            uint32_t last = (bits >> (valid - 1)) & 1u;
            for (int j = (int)valid; j < SP_PER; j++) bits = (bits & ~(1u << j)) | (last << j);
        }
        a.stencil[base / 8] = (uint8_t)bits;
    }
    const uint32_t valid_mask = base >= n ? 0u : (n - base >= SP_PER ? 0xffu : ((1u << (n - base)) - 1));
    const uint32_t yes_bits = bits & valid_mask;
    unsigned long long total;
    unsigned long long excl = block_exclusive_scan<SP_THREADS>((unsigned long long)__popc(yes_bits), ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    uint64_t yes_pos = s_prefix + excl;
    uint64_t no_pos = (base < n ? base : n) - yes_pos;
    for (int j = 0; j < SP_PER; j++) {
        if (!((valid_mask >> j) & 1u)) break;
        if ((yes_bits >> j) & 1u) {
            if (MODE == SPLIT_DICT) {
                const uint32_t c = (codes >> (2 * j)) & 3u;
                if (c) atomicOr(a.words + (yes_pos >> 4), c << (2 * (yes_pos & 15)));
            } else {
                st_elem<ES>(a.yes, yes_pos, v[j]);
            }
            ++yes_pos;
        } else {
            if (MODE != SPLIT_NOT_CONST) st_elem<ES>(a.no, no_pos, v[j]);
            ++no_pos;
        }
    }
    // the tile that ends the column reports the number of stencil-true elements
    if (base < n && base + SP_PER >= n) *a.yes_count = yes_pos;
}

// ------------------------------------------------------------------------------ merge
template <int ES, int MODE>
__global__ void __launch_bounds__(SP_THREADS)
k_merge(const uint8_t *__restrict__ stencil, uint64_t n, MergeArgs a, uint8_t *__restrict__ out, Lookback lb)
{
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0) s_tile = claim_tile(lb);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * SP_TILE + (uint64_t)threadIdx.x * SP_PER;
    const uint32_t valid_mask = base >= n ? 0u : (n - base >= SP_PER ? 0xffu : ((1u << (n - base)) - 1));
    const uint32_t bits = base < n ? ((uint32_t)__ldg(stencil + base / 8) & valid_mask) : 0u;
    unsigned long long total;
    unsigned long long excl = block_exclusive_scan<SP_THREADS>((unsigned long long)__popc(bits), ws, total);
    if (threadIdx.x < 32) {
        const unsigned long long e = lookback_exclusive(lb, tile, total);
        if (threadIdx.x == 0) s_prefix = e;
    }
    __syncthreads();
    if (base >= n) return;
    uint64_t top[4] = {0, 0, 0, 0};
    if (MODE != SPLIT_LOWER) {
#pragma unroll
        for (int k = 0; k < (MODE == SPLIT_DICT ? 4 : 1); k++) top[k] = ld_unaligned<ES>(a.top + k * ES);
    }
    uint64_t yes_pos = s_prefix + excl;
    uint64_t no_pos = base - yes_pos;
    uint64_t v[SP_PER];
#pragma unroll
    for (int j = 0; j < SP_PER; j++) {
        v[j] = 0;
        if (!((valid_mask >> j) & 1u)) continue;
        if ((bits >> j) & 1u) {
            if (yes_pos >= a.yes_cap) {
                atomicExch(a.error, (uint32_t)(-GTSC_ERR_FORMAT));
            } else if (MODE == SPLIT_DICT) {
                const uint32_t w = __ldg(a.words + (yes_pos >> 4));
                v[j] = top[(w >> (2 * (yes_pos & 15))) & 3u];
            } else {
                v[j] = ld_elem<ES>(a.yes, yes_pos);
            }
            ++yes_pos;
        } else {
            if (MODE == SPLIT_NOT_CONST) v[j] = top[0];
            else if (no_pos >= a.no_cap) atomicExch(a.error, (uint32_t)(-GTSC_ERR_FORMAT));
            else v[j] = ld_elem<ES>(a.no, no_pos);
            ++no_pos;
        }
    }
    store8<ES>(out, base, n, v);
}

}  // namespace

uint64_t split_tiles(uint64_t n) { return (n + SP_TILE - 1) / SP_TILE; }

void launch_split(int mode, const uint8_t *in, uint64_t n, int es, const SplitArgs &a, uint8_t *scratch,
                  cudaStream_t s)
{
    if (n == 0) return;
    const uint64_t tiles = split_tiles(n);
    GTSC_CUDA(cudaMemsetAsync(scratch, 0, lookback_zero_bytes(tiles), s));
    Lookback lb = lookback_at(scratch, tiles);
#define GTSC_SPLIT_CASE(E)                                                                             \
    switch (mode) {                                                                                    \
    case SPLIT_LOWER: k_split<E, SPLIT_LOWER><<<(unsigned)tiles, SP_THREADS, 0, s>>>(in, n, a, lb); break;          \
    case SPLIT_NOT_CONST: k_split<E, SPLIT_NOT_CONST><<<(unsigned)tiles, SP_THREADS, 0, s>>>(in, n, a, lb); break;  \
    default: k_split<E, SPLIT_DICT><<<(unsigned)tiles, SP_THREADS, 0, s>>>(in, n, a, lb); break;                   \
    }
    switch (es) {
    case 1: GTSC_SPLIT_CASE(1) break;
    case 2: GTSC_SPLIT_CASE(2) break;
    case 4: GTSC_SPLIT_CASE(4) break;
    default: GTSC_SPLIT_CASE(8) break;
    }
#undef GTSC_SPLIT_CASE
    GTSC_CUDA(cudaGetLastError());
}

void launch_merge(int mode, const uint8_t *stencil, uint64_t n, int es, const MergeArgs &a, uint8_t *out,
                  uint8_t *scratch, cudaStream_t s)
{
    if (n == 0) return;
    const uint64_t tiles = split_tiles(n);
    GTSC_CUDA(cudaMemsetAsync(scratch, 0, lookback_zero_bytes(tiles), s));
    Lookback lb = lookback_at(scratch, tiles);
#define GTSC_MERGE_CASE(E)                                                                                       \
    switch (mode) {                                                                                              \
    case SPLIT_LOWER: k_merge<E, SPLIT_LOWER><<<(unsigned)tiles, SP_THREADS, 0, s>>>(stencil, n, a, out, lb); break;         \
    case SPLIT_NOT_CONST: k_merge<E, SPLIT_NOT_CONST><<<(unsigned)tiles, SP_THREADS, 0, s>>>(stencil, n, a, out, lb); break; \
    default: k_merge<E, SPLIT_DICT><<<(unsigned)tiles, SP_THREADS, 0, s>>>(stencil, n, a, out, lb); break;                  \
    }
    switch (es) {
    case 1: GTSC_MERGE_CASE(1) break;
    case 2: GTSC_MERGE_CASE(2) break;
    case 4: GTSC_MERGE_CASE(4) break;
    default: GTSC_MERGE_CASE(8) break;
    }
#undef GTSC_MERGE_CASE
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
