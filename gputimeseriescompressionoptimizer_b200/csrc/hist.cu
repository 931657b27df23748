// hist.cu -- exact value histogram and top-k (Histogram::GetMostFrequent,
// util/histogram/histogram.cpp:28-35).
//
// The reference sorts the whole column (thrust::sort), counts bins with inner_product +
// reduce_by_key and sorts the bins by count (thrust_sparse_histogram.cu:19-69,
// most_frequent.cu:10-26).  Here:
//   k_hist   -- each block aggregates its slice of the column in a 2048-entry shared-memory hash
//               table (64-bit CAS on keys, counts by shared atomics); keys that do not fit go
//               straight to a global open-addressing table, and the block flushes its table there
//               at the end.  NaN elements never merge (they are singleton bins in the reference),
//               so each block only keeps the 4 smallest NaN sort keys it saw.
//   k_topk   -- blocks scan the global table keeping the best 4 entries by (count desc, value
//               asc in sort order) in registers; a final 1-block pass merges the block lists, the
//               NaN candidates and the one key value the table cannot hold.
// Ties follow the reference's stable radix sort of (ascending) bins: count desc, then value asc.
#include "kernels.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int H_THREADS = 256;
constexpr int SM_CAP = 2048;
constexpr unsigned long long EMPTY = ~0ull;
constexpr int SM_PROBE = 8;

__device__ __forceinline__ uint64_t hash64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

struct Cand {
    unsigned long long key;  // order key of the value
    unsigned long long bits; // raw value bits
    unsigned int count;
};

// a ranks before b: more occurrences, then smaller value
__device__ __forceinline__ bool better(const Cand &a, const Cand &b)
{
    return a.count > b.count || (a.count == b.count && a.count != 0 && a.key < b.key);
}

__device__ __forceinline__ void push4(Cand *list, const Cand &c)
{
    if (!better(c, list[3])) return;
    list[3] = c;
#pragma unroll
    for (int i = 3; i > 0; i--)
        if (better(list[i], list[i - 1])) {
            Cand t = list[i];
            list[i] = list[i - 1];
            list[i - 1] = t;
        }
}

__device__ bool global_insert(const HistTable &t, unsigned long long key, unsigned int c)
{
    if (key == EMPTY) {
        atomicAdd(t.special, c);
        return true;
    }
    const uint64_t mask = t.cap - 1;
    uint64_t h = hash64(key) & mask;
    for (uint64_t probe = 0; probe < t.cap; probe++) {
        unsigned long long prev = atomicCAS(t.keys + h, EMPTY, key);
        if (prev == EMPTY || prev == key) {
            atomicAdd(t.counts + h, c);
            return true;
        }
        h = (h + 1) & mask;
        if (probe > 4096) break;
    }
    atomicExch(t.overflow, 1u);
    return false;
}

template <int ES>
__global__ void __launch_bounds__(H_THREADS)
k_hist(const uint8_t *__restrict__ in, uint64_t n, Order o, HistTable t)
{
    __shared__ unsigned long long skeys[SM_CAP];
    __shared__ unsigned int scounts[SM_CAP];
    __shared__ unsigned long long snan[H_THREADS / 32][4];
    for (int i = threadIdx.x; i < SM_CAP; i += H_THREADS) {
        skeys[i] = EMPTY;
        scounts[i] = 0;
    }
    __syncthreads();
    unsigned long long nan_min[4] = {EMPTY, EMPTY, EMPTY, EMPTY};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned long long key = ld_elem<ES>(in, i);
        if (is_nan_bits(key, o)) {
            unsigned long long k = order_key(key, ES, o);
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (k < nan_min[j]) { unsigned long long tmp = nan_min[j]; nan_min[j] = k; k = tmp; }
            continue;
        }
        bool done = false;
        if (key != EMPTY) {
            uint32_t h = (uint32_t)hash64(key) & (SM_CAP - 1);
            for (int p = 0; p < SM_PROBE; p++) {
                unsigned long long prev = atomicCAS(&skeys[h], EMPTY, key);
                if (prev == EMPTY || prev == key) {
                    atomicAdd(&scounts[h], 1u);
                    done = true;
                    break;
                }
                h = (h + 1) & (SM_CAP - 1);
            }
        }
        if (!done) global_insert(t, key, 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SM_CAP; i += H_THREADS)
        if (skeys[i] != EMPTY) global_insert(t, skeys[i], scounts[i]);
    // the block's 4 smallest NaN keys
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long other[4];
#pragma unroll
        for (int j = 0; j < 4; j++) other[j] = __shfl_xor_sync(0xffffffffu, nan_min[j], off);
        unsigned long long merged[4];
        int a = 0, b = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (nan_min[a] <= other[b]) merged[j] = nan_min[a++];
            else merged[j] = other[b++];
        }
#pragma unroll
        for (int j = 0; j < 4; j++) nan_min[j] = merged[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int j = 0; j < 4; j++) snan[warp][j] = nan_min[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long best[4] = {EMPTY, EMPTY, EMPTY, EMPTY};
        for (int w = 0; w < H_THREADS / 32; w++)
            for (int j = 0; j < 4; j++) {
                unsigned long long k = snan[w][j];
                for (int q = 0; q < 4; q++)
                    if (k < best[q]) { unsigned long long tmp = best[q]; best[q] = k; k = tmp; }
            }
        for (int j = 0; j < 4; j++) t.nan_keys[4 * blockIdx.x + j] = best[j];
    }
}

// per-block best 4 of the global table
__global__ void __launch_bounds__(H_THREADS)
k_topk_partial(HistTable t, int es, Order o, Cand *partial)
{
    Cand list[4];
    for (int j = 0; j < 4; j++) list[j] = Cand{EMPTY, 0, 0};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < t.cap; i += stride) {
        const unsigned long long k = t.keys[i];
        if (k == EMPTY) continue;
        push4(list, Cand{order_key(k, es, o), k, t.counts[i]});
    }
    __shared__ Cand s[H_THREADS * 4];
    for (int j = 0; j < 4; j++) s[threadIdx.x * 4 + j] = list[j];
    __syncthreads();
    for (int width = H_THREADS / 2; width > 0; width >>= 1) {
        if (threadIdx.x < width)
            for (int j = 0; j < 4; j++) {
                Cand c = s[(threadIdx.x + width) * 4 + j];
                Cand *mine = &s[threadIdx.x * 4];
                if (better(c, mine[3])) {
                    Cand l[4] = {mine[0], mine[1], mine[2], mine[3]};
                    push4(l, c);
                    for (int q = 0; q < 4; q++) mine[q] = l[q];
                }
            }
        __syncthreads();
    }
    if (threadIdx.x < 4) partial[blockIdx.x * 4 + threadIdx.x] = s[threadIdx.x];
}

// merge: block partials, NaN singletons, the special key; writes k values (es bytes each)
__global__ void k_topk_final(HistTable t, const Cand *partial, int nparts, int nnan, int es, Order o, int k,
                             uint8_t *top_out, unsigned long long *count_out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Cand list[4];
    for (int j = 0; j < 4; j++) list[j] = Cand{EMPTY, 0, 0};
    for (int p = 0; p < nparts * 4; p++)
        if (partial[p].count) push4(list, partial[p]);
    const unsigned int sp = *t.special;
    if (sp) push4(list, Cand{order_key(EMPTY, es, o), EMPTY, sp});
    for (int p = 0; p < nnan * 4; p++) {
        unsigned long long key = t.nan_keys[p];
        if (key == EMPTY) continue;
        push4(list, Cand{key, order_unkey(key, es, o), 1u});
    }
    for (int j = 0; j < k; j++) {
        const unsigned long long bits = list[j].count ? list[j].bits : 0ull;  // unused slots are 0
        for (int b = 0; b < es; b++) top_out[j * es + b] = (uint8_t)(bits >> (8 * b));
        if (count_out) count_out[j] = list[j].count;
    }
}

}  // namespace

uint64_t hist_cap_for(uint64_t n, bool full)
{
    uint64_t want = 2 * n + 64;
    uint64_t cap = 1024;
    while (cap < want) cap <<= 1;
    const uint64_t small = 1ull << 22;
    return (!full && cap > small) ? small : cap;
}

int hist_grid(uint64_t n)
{
    uint64_t b = (n + H_THREADS * 16 - 1) / (H_THREADS * 16);
    uint64_t cap = (uint64_t)sm_count() * 2;
    if (b > cap) b = cap;
    return (int)(b ? b : 1);
}

uint64_t hist_scratch_bytes(uint64_t cap, int grid)
{
    return 8 * cap + 4 * cap + 32 + 32ull * grid + sizeof(unsigned long long) * 3 * 4 * 256 + 64;
}

HistTable hist_table_at(uint8_t *scratch, uint64_t cap, int grid)
{
    HistTable t;
    t.cap = cap;
    t.keys = (unsigned long long *)scratch;
    t.counts = (unsigned int *)(scratch + 8 * cap);
    uint8_t *p = scratch + 12 * cap;
    t.special = (unsigned int *)p;
    t.overflow = (unsigned int *)(p + 4);
    t.nan_keys = (unsigned long long *)(p + 32);
    t.partial = p + 32 + 32ull * grid;
    return t;
}

void launch_hist_topk(const uint8_t *in, uint64_t n, int es, Order o, int k, const HistTable &t, int grid,
                      uint8_t *top_out, unsigned long long *count_out, cudaStream_t s)
{
    GTSC_CUDA(cudaMemsetAsync(t.keys, 0xff, 8 * t.cap, s));
    GTSC_CUDA(cudaMemsetAsync(t.counts, 0, 4 * t.cap + 32, s));
    if (n) {
        switch (es) {
        case 1: k_hist<1><<<grid, H_THREADS, 0, s>>>(in, n, o, t); break;
        case 2: k_hist<2><<<grid, H_THREADS, 0, s>>>(in, n, o, t); break;
        case 4: k_hist<4><<<grid, H_THREADS, 0, s>>>(in, n, o, t); break;
        default: k_hist<8><<<grid, H_THREADS, 0, s>>>(in, n, o, t); break;
        }
        GTSC_CUDA(cudaGetLastError());
    }
    int pg = (int)((t.cap + H_THREADS * 8 - 1) / (H_THREADS * 8));
    if (pg > 256) pg = 256;
    Cand *partial = (Cand *)t.partial;
    k_topk_partial<<<pg, H_THREADS, 0, s>>>(t, es, o, partial);
    GTSC_CUDA(cudaGetLastError());
    k_topk_final<<<1, 32, 0, s>>>(t, partial, pg, n ? grid : 0, es, o, k, top_out, count_out);
    GTSC_CUDA(cudaGetLastError());
}

}  // namespace gtsc
