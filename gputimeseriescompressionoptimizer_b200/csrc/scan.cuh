// scan.cuh -- single-pass device-wide prefix scans by decoupled look-back, written for sm_100a.
//
// A kernel processes tiles in the order it claims them from a global counter (so every tile's
// predecessors were claimed earlier and make progress).  Thread 0 of a tile publishes the tile's
// aggregate (flag 1), walks back over the predecessors' flags, adds their aggregates until it finds
// an inclusive prefix (flag 2), then publishes its own inclusive prefix.  Flags and values are
// separate words ordered with st.release / ld.acquire at gpu scope.  Every wait is bounded: after
// kSpinLimit polls the tile records GTSC_ERR_TIMEOUT in *error and proceeds with a wrong prefix,
// so a broken predecessor can never hang the GPU; the host turns the error word into a status.
//
// Values are 64-bit and combine by wrapping addition, which also serves 8/16/32-bit wrapping
// arithmetic (the low bits of a 64-bit wrapping sum are the narrow wrapping sum).
#pragma once

#include "common.cuh"

namespace gtsc {

constexpr uint32_t kSpinLimit = 1u << 22;  // ~0.3 s of polling with back-off

struct Lookback {
    uint32_t *counter;             // tile claim counter (zeroed before launch)
    uint32_t *flags;               // per tile: 0 none, 1 aggregate, 2 inclusive prefix (zeroed)
    unsigned long long *agg;       // per tile aggregate
    unsigned long long *pre;       // per tile inclusive prefix
    uint32_t *error;               // set to a gtsc_status on timeout (zeroed)
};

// bytes of scratch for `tiles` tiles; layout: counter, error, pad, flags[tiles], agg[tiles], pre[tiles]
__host__ __device__ inline uint64_t lookback_bytes(uint64_t tiles)
{
    return 16 + ((4 * tiles + 15) & ~15ull) + 16 * tiles;
}
// bytes that must be zeroed before each launch (counter, error and the flags)
__host__ __device__ inline uint64_t lookback_zero_bytes(uint64_t tiles) { return 16 + 4 * tiles; }

__host__ __device__ inline Lookback lookback_at(uint8_t *scratch, uint64_t tiles)
{
    Lookback l;
    l.counter = (uint32_t *)scratch;
    l.error = (uint32_t *)(scratch + 4);
    l.flags = (uint32_t *)(scratch + 16);
    uint8_t *v = scratch + 16 + ((4 * tiles + 15) & ~15ull);
    l.agg = (unsigned long long *)v;
    l.pre = (unsigned long long *)(v + 8 * tiles);
    return l;
}

__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Claims the next tile id (one thread per block; broadcast through shared memory by the caller).
__device__ __forceinline__ uint32_t claim_tile(const Lookback &l) { return atomicAdd(l.counter, 1u); }

// Called by ONE thread of the block that owns `tile`: publishes the tile aggregate and returns
// the exclusive prefix (wrapping sum of all earlier tiles).
__device__ inline unsigned long long lookback_exclusive(const Lookback &l, uint32_t tile, unsigned long long tile_agg)
{
    if (tile == 0) {
        l.pre[0] = tile_agg;
        st_release_u32(&l.flags[0], 2u);
        return 0ull;
    }
    l.agg[tile] = tile_agg;
    st_release_u32(&l.flags[tile], 1u);
    unsigned long long excl = 0;
    int64_t t = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (t >= 0) {
        uint32_t f = ld_acquire_u32(&l.flags[t]);
        if (f == 2u) {
            excl += ld_relaxed_u64(&l.pre[t]);
            break;
        }
        if (f == 1u) {
            excl += ld_relaxed_u64(&l.agg[t]);
            --t;
            continue;
        }
        if (++spins > kSpinLimit) {
            atomicExch(l.error, (uint32_t)(-GTSC_ERR_TIMEOUT));
            break;
        }
        __nanosleep(spins < 64 ? 32 : 256);
    }
    l.pre[tile] = excl + tile_agg;
    st_release_u32(&l.flags[tile], 2u);
    return excl;
}

// Block-wide exclusive scan (wrapping add) of one 64-bit value per thread; also returns the block
// total.  `ws` must hold 32 entries of shared memory.  All threads of the block must call it.
template <int THREADS>
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long *ws,
                                                                   unsigned long long &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < THREADS / 32 ? ws[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < THREADS / 32) ws[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    total = ws[THREADS / 32 - 1];
    unsigned long long base = warp ? ws[warp - 1] : 0ull;
    unsigned long long r = base + x - v;
    __syncthreads();
    return r;
}

}  // namespace gtsc
