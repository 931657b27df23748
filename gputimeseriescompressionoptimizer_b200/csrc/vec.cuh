// vec.cuh -- vectorised element access for byte buffers of 1/2/4/8-byte elements.
#pragma once

#include "common.cuh"

namespace gtsc {

// Read-only loads.  Data that earlier work of the same kernel may have written must not be read
// through the non-coherent read-only path (ld.global.nc is only defined for data that no thread
// writes while the kernel runs).  The batch engine's translation units hold persistent kernels in
// which later passes read what earlier passes wrote, so they define GTSC_COHERENT_LOADS before
// including this header and get plain (L1-cached, coherent after an acquire) loads instead.
// (internal linkage: the two definitions never meet across translation units)
#ifdef GTSC_COHERENT_LOADS
template <class T>
static __device__ __forceinline__ T ldg(const T *p)
{
    return *p;
}
#else
template <class T>
static __device__ __forceinline__ T ldg(const T *p)
{
    return __ldg(p);
}
#endif

// Element j (of width ES <= 4) of a 16-byte chunk; ES == 8 is specialised below.
template <int ES>
__device__ __forceinline__ uint64_t chunk_elem(const uint4 &c, int j)
{
    const int word = (j * ES) >> 2;
    const uint32_t w = word == 0 ? c.x : word == 1 ? c.y : word == 2 ? c.z : c.w;
    if (ES == 4) return w;
    const int sh = ((j * ES) & 3) * 8;
    if (ES == 2) return (w >> sh) & 0xffffu;
    return (w >> sh) & 0xffu;
}

template <>
__device__ __forceinline__ uint64_t chunk_elem<8>(const uint4 &c, int j)
{
    return j == 0 ? ((uint64_t)c.y << 32 | c.x) : ((uint64_t)c.w << 32 | c.z);
}

// Scalar load of element i (raw bits, zero-extended).
template <int ES>
__device__ __forceinline__ uint64_t ld_elem(const uint8_t *p, uint64_t i)
{
    if (ES == 1) return ldg(p + i);
    if (ES == 2) return ldg((const unsigned short *)p + i);
    if (ES == 4) return ldg((const unsigned int *)p + i);
    return ldg((const unsigned long long *)p + i);
}

// Little-endian load of an ES-byte value at any address (metadata fields inside a blob).
template <int ES>
__device__ __forceinline__ uint64_t ld_unaligned(const uint8_t *p)
{
    uint64_t v = 0;
#pragma unroll
    for (int k = 0; k < ES; k++) v |= (uint64_t)ldg(p + k) << (8 * k);
    return v;
}

template <int ES>
__device__ __forceinline__ void st_elem(uint8_t *p, uint64_t i, uint64_t v)
{
    if (ES == 1) p[i] = (uint8_t)v;
    else if (ES == 2) ((uint16_t *)p)[i] = (uint16_t)v;
    else if (ES == 4) ((uint32_t *)p)[i] = (uint32_t)v;
    else ((unsigned long long *)p)[i] = v;
}

__device__ __forceinline__ uint4 ld_chunk(const uint8_t *p)  // p 16-byte aligned
{
    return ldg((const uint4 *)p);
}

// Pack element values into a 16-byte chunk.
template <int ES>
__device__ __forceinline__ uint4 make_chunk(const uint64_t *v)
{
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 16 / ES; j++) {
        if constexpr (ES == 8) {
            w[2 * j] = (uint32_t)v[j];
            w[2 * j + 1] = (uint32_t)(v[j] >> 32);
        } else if constexpr (ES == 4) {
            w[j] = (uint32_t)v[j];
        } else {
            const int word = (j * ES) >> 2, sh = ((j * ES) & 3) * 8;
            constexpr uint32_t m = (1u << (8 * ES)) - 1;
            w[word] |= ((uint32_t)v[j] & m) << sh;
        }
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// Byte-stream reader for a stream that starts at an arbitrary address: loads the 32-bit word
// that covers stream bits [32*w - off_bits, ...) from the 4-byte aligned base, zero past the end.
struct StreamReader {
    const uint32_t *base;   // 4-byte aligned
    uint64_t nbytes;        // bytes valid from base
    __device__ __forceinline__ uint32_t word(uint64_t w) const
    {
        uint64_t b = 4 * w;
        if (b + 4 <= nbytes) return ldg(base + w);
        uint32_t r = 0;
        const uint8_t *p = (const uint8_t *)base;
        for (int k = 0; k < 4; k++)
            if (b + k < nbytes) r |= (uint32_t)p[b + k] << (8 * k);
        return r;
    }
};

}  // namespace gtsc
