// common.cuh -- shared device helpers and host plumbing of libgtsc (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gtsc.h"

namespace gtsc {

// ---------------------------------------------------------------------------------- errors

struct Error : std::runtime_error {
    gtsc_status code;
    Error(gtsc_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(gtsc_status code, const std::string &msg);
void cuda_check(cudaError_t e, const char *what);
#define GTSC_CUDA(x) ::gtsc::cuda_check((x), #x)

void set_last_error(const std::string &m);

// ---------------------------------------------------------------------------------- types

inline int dtype_size(int dt)
{
    switch (dt) {
    case GTSC_CHAR: return 1;
    case GTSC_SHORT: return 2;
    case GTSC_INT: case GTSC_FLOAT: return 4;
    case GTSC_TIME: case GTSC_DOUBLE: return 8;
    default: return 0;
    }
}
inline bool is_fp(int dt) { return dt == GTSC_FLOAT || dt == GTSC_DOUBLE; }

// Order used by min/max reductions: signed integer of the element width, or IEEE order.
enum Order : int { ORD_INT = 0, ORD_F32 = 1, ORD_F64 = 2 };
inline Order native_order(int dt)
{
    return dt == GTSC_FLOAT ? ORD_F32 : dt == GTSC_DOUBLE ? ORD_F64 : ORD_INT;
}

// ---------------------------------------------------------------------------------- buffers

// Device allocation released with cudaFreeAsync on the stream it was allocated on, unless its
// ownership was handed over (disown) to a C caller.
struct DevMem {
    uint8_t *p = nullptr;
    cudaStream_t s = nullptr;
    bool owned = true;
    ~DevMem()
    {
        if (p && owned) cudaFreeAsync(p, s);
    }
};

// Shared handle of a device buffer.
struct DevBuf {
    std::shared_ptr<DevMem> m;
    uint64_t bytes = 0;
    uint8_t *get() const { return m ? m->p : nullptr; }
    // free on the legacy stream instead of the allocating one (for buffers that may outlive that
    // stream; the owner synchronises the device before releasing them)
    void release_on_default_stream()
    {
        if (m) m->s = nullptr;
    }
    // give up ownership (the caller frees the pointer); returns it
    uint8_t *disown()
    {
        if (!m) return nullptr;
        m->owned = false;
        return m->p;
    }
};
DevBuf dev_alloc(uint64_t bytes, cudaStream_t s);

// Non-owning view of device bytes.
struct View {
    const uint8_t *ptr = nullptr;
    uint64_t bytes = 0;
    View() = default;
    View(const void *p, uint64_t b) : ptr((const uint8_t *)p), bytes(b) {}
    View(const DevBuf &b) : ptr(b.get()), bytes(b.bytes) {}
};

using Parts = std::vector<DevBuf>;

int sm_count();

// Host copy of a few device bytes (synchronising the stream).
void d2h(void *dst, const void *src, uint64_t bytes, cudaStream_t s);

// ---------------------------------------------------------------------------------- device

#define GTSC_HD __host__ __device__ __forceinline__

// Monotone 64-bit key of an element's raw bits: signed order for integers of width es,
// IEEE "twiddle" order for floats (-0 sorts before +0).
GTSC_HD uint64_t order_key(uint64_t u, int es, Order o)
{
    if (o == ORD_F32) {
        uint32_t v = (uint32_t)u;
        return (v & 0x80000000u) ? (uint32_t)~v : (v | 0x80000000u);
    }
    if (o == ORD_F64) return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
    int sh = 64 - 8 * es;
    int64_t s = (int64_t)(u << sh) >> sh;  // sign-extend
    return (uint64_t)s ^ 0x8000000000000000ull;
}
GTSC_HD uint64_t order_unkey(uint64_t k, int es, Order o)
{
    if (o == ORD_F32) {
        uint32_t v = (uint32_t)k;
        return (v & 0x80000000u) ? (v & 0x7fffffffu) : (uint32_t)~v;
    }
    if (o == ORD_F64) return (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    uint64_t s = k ^ 0x8000000000000000ull;
    return es == 8 ? s : (s & ((1ull << (8 * es)) - 1));
}
GTSC_HD bool is_nan_bits(uint64_t u, Order o)
{
    if (o == ORD_F32) return ((u >> 23) & 0xff) == 0xff && (u & 0x7fffff) != 0;
    if (o == ORD_F64) return ((u >> 52) & 0x7ff) == 0x7ff && (u & 0xfffffffffffffull) != 0;
    return false;
}
GTSC_HD int64_t sext(uint64_t u, int es)
{
    int sh = 64 - 8 * es;
    return (int64_t)(u << sh) >> sh;
}

#ifdef __CUDACC__
// `a < b` in the element's own arithmetic (IEEE compare for floats: -0 < +0 is false, NaN false)
__device__ __forceinline__ bool lt_native(uint64_t a, uint64_t b, int es, Order o)
{
    if (o == ORD_F32) return __uint_as_float((uint32_t)a) < __uint_as_float((uint32_t)b);
    if (o == ORD_F64) return __longlong_as_double((long long)a) < __longlong_as_double((long long)b);
    return sext(a, es) < sext(b, es);
}
#endif

// BITLEN<T>(min, max) for signed integer T (core/cuda_macros.cuh:168-175)
GTSC_HD int bitlen_signed(int64_t mn, int64_t mx, int es)
{
    if (mn < 0) return 8 * es;
#ifdef __CUDA_ARCH__
    return mx == 0 ? 1 : 64 - __clzll((unsigned long long)mx);
#else
    int r = 0;
    while (mx >>= 1) r++;
    return r + 1;
#endif
}

// Result of the min/max pass: bits of the smallest and largest element in the given order, the
// smallest stored complemented so that both reduce with atomicMax from a zeroed buffer.
struct MinMaxAcc {
    unsigned long long nkmin;  // ~key(min); 0 = nothing seen
    unsigned long long kmax;   // key(max)
};

}  // namespace gtsc
