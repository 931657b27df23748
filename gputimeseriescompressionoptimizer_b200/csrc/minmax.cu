// minmax.cu -- single-pass min/max over a column (CudaArrayStatistics::MinMax,
// util/statistics/cuda_array_statistics.cu:20-28, which runs thrust::minmax_element).
//
// HBM-bound: every element is read once with 16-byte loads; each block folds its keys with warp
// shuffles and issues two 64-bit atomicMax into a zeroed accumulator.
#include "kernels.hpp"
#include "vec.cuh"

namespace gtsc {

namespace {

constexpr int MM_THREADS = 256;

__device__ __forceinline__ void fold(uint64_t u, int es, Order o, uint64_t &kmin, uint64_t &kmax)
{
    if (is_nan_bits(u, o)) return;
    uint64_t k = order_key(u, es, o);
    kmin = k < kmin ? k : kmin;
    kmax = k > kmax ? k : kmax;
}

template <int ES>
__global__ void __launch_bounds__(MM_THREADS)
k_minmax(const uint8_t *__restrict__ in, uint64_t n, uint64_t head, Order o, MinMaxAcc *acc)
{
    uint64_t kmin = ~0ull, kmax = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // unaligned head elements, then 16-byte chunks, then the tail
    if (gtid < head && gtid < n) fold(ld_elem<ES>(in, gtid), ES, o, kmin, kmax);
    const uint8_t *body = in + head * ES;
    const uint64_t nb = n > head ? n - head : 0;
    const uint64_t nchunks = nb * ES / 16;
    for (uint64_t c = gtid; c < nchunks; c += stride) {
        uint4 v = ld_chunk(body + 16 * c);
#pragma unroll
        for (int j = 0; j < 16 / ES; j++) fold(chunk_elem<ES>(v, j), ES, o, kmin, kmax);
    }
    const uint64_t done = nchunks * 16 / ES;
    if (gtid < nb - done) fold(ld_elem<ES>(body, done + gtid), ES, o, kmin, kmax);

    for (int off = 16; off > 0; off >>= 1) {
        uint64_t a = __shfl_xor_sync(0xffffffffu, kmin, off);
        uint64_t b = __shfl_xor_sync(0xffffffffu, kmax, off);
        kmin = a < kmin ? a : kmin;
        kmax = b > kmax ? b : kmax;
    }
    __shared__ uint64_t smin[MM_THREADS / 32], smax[MM_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { smin[warp] = kmin; smax[warp] = kmax; }
    __syncthreads();
    if (warp == 0) {
        kmin = lane < MM_THREADS / 32 ? smin[lane] : ~0ull;
        kmax = lane < MM_THREADS / 32 ? smax[lane] : 0;
        for (int off = 4; off > 0; off >>= 1) {
            uint64_t a = __shfl_xor_sync(0xffffffffu, kmin, off);
            uint64_t b = __shfl_xor_sync(0xffffffffu, kmax, off);
            kmin = a < kmin ? a : kmin;
            kmax = b > kmax ? b : kmax;
        }
        if (lane == 0) {
            if (kmin != ~0ull) atomicMax(&acc->nkmin, (unsigned long long)~kmin);
            if (kmax != 0) atomicMax(&acc->kmax, (unsigned long long)kmax);
        }
    }
}

}  // namespace

void launch_minmax(const uint8_t *in, uint64_t n, int es, Order o, MinMaxAcc *acc, cudaStream_t s)
{
    if (n == 0) return;
    uint64_t mis = (uintptr_t)in & 15;
    uint64_t head = mis ? (16 - mis) / es : 0;
    if (head > n) head = n;
    uint64_t work = (n * es) / 16 + 1;
    uint64_t blocks = (work + MM_THREADS - 1) / MM_THREADS;
    uint64_t cap = (uint64_t)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    switch (es) {
    case 1: k_minmax<1><<<blocks, MM_THREADS, 0, s>>>(in, n, head, o, acc); break;
    case 2: k_minmax<2><<<blocks, MM_THREADS, 0, s>>>(in, n, head, o, acc); break;
    case 4: k_minmax<4><<<blocks, MM_THREADS, 0, s>>>(in, n, head, o, acc); break;
    default: k_minmax<8><<<blocks, MM_THREADS, 0, s>>>(in, n, head, o, acc); break;
    }
    GTSC_CUDA(cudaGetLastError());
}

bool minmax_result(const MinMaxAcc &acc, int es, Order o, uint64_t *mn, uint64_t *mx)
{
    if (acc.nkmin == 0 && acc.kmax == 0) return false;
    *mn = order_unkey(~(uint64_t)acc.nkmin, es, o);
    *mx = order_unkey(acc.kmax, es, o);
    return true;
}

}  // namespace gtsc
