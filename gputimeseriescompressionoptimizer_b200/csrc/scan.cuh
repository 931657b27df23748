// scan.cuh -- single-pass device-wide prefix scans by decoupled look-back, written for sm_100a.
//
// A kernel processes tiles in the order it claims them from a global counter (so every tile's
// predecessors were claimed earlier and make progress).  One warp of a tile publishes the tile's
// aggregate (flag 1), reads its predecessors' descriptors 128 at a time, adds their aggregates
// until it finds an inclusive prefix (flag 2), then publishes its own inclusive prefix.  A descriptor is
// two relaxed gpu-scope 64-bit words that both carry the flag, so a reader needs no acquire chain.
// Every wait is bounded: after kSpinLimit polls, or as soon as another tile has recorded an error,
// the tile records GTSC_ERR_TIMEOUT in *error and proceeds with a wrong prefix, so a broken
// predecessor can never hang the GPU; the host turns the error word into a status.
//
// Values are 64-bit and combine by wrapping addition, which also serves 8/16/32-bit wrapping
// arithmetic (the low bits of a 64-bit wrapping sum are the narrow wrapping sum).
#pragma once

#include "common.cuh"

namespace gtsc {

constexpr uint32_t kSpinLimit = 1u << 22;  // ~0.3 s of polling with back-off

struct Lookback {
    uint32_t *counter;             // tile claim counter (zeroed before launch)
    uint32_t *error;               // set to a gtsc_status on timeout (zeroed)
    unsigned long long *desc;      // per tile two words: flag 0 none, 1 aggregate, 2 inclusive (zeroed)
};

// bytes of scratch for `tiles` tiles; layout: counter, error, pad, then per tile two 64-bit
// descriptor words (word 0 = flag << 32 | low half of the value, word 1 = flag << 32 | high half)
__host__ __device__ constexpr uint64_t lookback_bytes(uint64_t tiles) { return 16 + 16 * tiles; }
// bytes that must be zeroed before each launch (counter, error and the descriptors)
__host__ __device__ constexpr uint64_t lookback_zero_bytes(uint64_t tiles) { return 16 + 16 * tiles; }

__host__ __device__ inline Lookback lookback_at(uint8_t *scratch, uint64_t tiles)
{
    Lookback l;
    l.counter = (uint32_t *)scratch;
    l.error = (uint32_t *)(scratch + 4);
    l.desc = (unsigned long long *)(scratch + 16);
    (void)tiles;
    return l;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Claims the next tile id (one thread per block; broadcast through shared memory by the caller).
__device__ __forceinline__ uint32_t claim_tile(const Lookback &l) { return atomicAdd(l.counter, 1u); }

// A descriptor is published as two words that each carry the flag, so a reader that sees the
// same flag in both has a consistent value without any ordering between the stores.
__device__ __forceinline__ void lookback_publish(const Lookback &l, uint32_t tile, uint32_t flag,
                                                 unsigned long long v)
{
    const unsigned long long f = (unsigned long long)flag << 32;
    st_relaxed_u64(l.desc + 2 * (uint64_t)tile, f | (v & 0xffffffffull));
    st_relaxed_u64(l.desc + 2 * (uint64_t)tile + 1, f | (v >> 32));
}

constexpr int kLookbackPerLane = 4;  // descriptors read by each lane per round trip (window 128)

// Called by all 32 lanes of ONE warp of the block that owns `tile` (the same tile_agg in every
// lane): publishes the tile aggregate and returns the exclusive prefix (wrapping sum of all
// earlier tiles) in every lane.  The warp reads a window of 128 predecessors per round trip (lane
// k reads tiles base - 4k .. base - 4k - 3, nearest first), sums the window up to its nearest
// inclusive prefix (or wholly when it holds only aggregates, then moves 128 tiles back), and waits
// only while a tile nearer than that prefix has published nothing.
__device__ inline unsigned long long lookback_exclusive(const Lookback &l, uint32_t tile, unsigned long long tile_agg)
{
    constexpr int PL = kLookbackPerLane;
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) lookback_publish(l, 0, 2u, tile_agg);
        return 0ull;
    }
    if (lane == 0) lookback_publish(l, tile, 1u, tile_agg);
    unsigned long long excl = 0;
    int64_t base = (int64_t)tile - 1;
    uint32_t spins = 0;
    bool gave_up = false;
    while (true) {
        uint32_t flag[PL];
        unsigned long long v[PL];
#pragma unroll
        for (int j = 0; j < PL; j++) {
            const int64_t idx = base - (int64_t)(PL * lane + j);
            flag[j] = 2u;
            v[j] = 0;
            if (idx >= 0) {
                const unsigned long long w0 = ld_relaxed_u64(l.desc + 2 * idx);
                const unsigned long long w1 = ld_relaxed_u64(l.desc + 2 * idx + 1);
                const uint32_t f0 = (uint32_t)(w0 >> 32), f1 = (uint32_t)(w1 >> 32);
                flag[j] = f0 == f1 ? f0 : 0u;
                v[j] = (w0 & 0xffffffffull) | (w1 << 32);
            }
            if (gave_up && flag[j] == 0u) {  // bounded wait ran out: treat as an empty prefix
                flag[j] = 2u;
                v[j] = 0;
            }
        }
        // this lane's nearest inclusive and nearest unpublished slot (PL = none)
        int inc = PL, inv = PL;
#pragma unroll
        for (int j = PL - 1; j >= 0; j--) {
            if (flag[j] == 2u) inc = j;
            if (flag[j] == 0u) inv = j;
        }
        const unsigned inc_lanes = __ballot_sync(0xffffffffu, inc < PL);
        const unsigned inv_lanes = __ballot_sync(0xffffffffu, inv < PL);
        const int L_inc = inc_lanes ? __ffs(inc_lanes) - 1 : 32;
        const int inc_pos = L_inc < 32 ? PL * L_inc + __shfl_sync(0xffffffffu, inc, L_inc & 31) : 32 * PL;
        const int L_inv = inv_lanes ? __ffs(inv_lanes) - 1 : 32;
        const int inv_pos = L_inv < 32 ? PL * L_inv + __shfl_sync(0xffffffffu, inv, L_inv & 31) : 32 * PL;
        if (inv_pos < inc_pos) {  // a nearer tile has not published yet
            ++spins;
            const bool err = (spins & 63u) == 0 && *(volatile uint32_t *)l.error != 0u;
            if (spins > kSpinLimit || __any_sync(0xffffffffu, err)) {
                if (lane == 0) atomicExch(l.error, (uint32_t)(-GTSC_ERR_TIMEOUT));
                gave_up = true;
            } else {
                __nanosleep(spins < 64 ? 32 : 256);
            }
            continue;
        }
        unsigned long long sum = 0;
#pragma unroll
        for (int j = 0; j < PL; j++)
            if (PL * lane + j <= inc_pos) sum += v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        excl += sum;
        if (inc_pos < 32 * PL) break;
        base -= 32 * PL;
    }
    if (lane == 0) lookback_publish(l, tile, 2u, excl + tile_agg);
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
