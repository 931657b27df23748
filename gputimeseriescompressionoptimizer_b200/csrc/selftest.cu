// selftest.cu -- gtsc_selftest_lookback_timeout: the bounded wait of the decoupled look-back
// (scan.cuh) run against a predecessor tile that never publishes.
#include "scan.cuh"

#include <chrono>

namespace gtsc {
namespace {

// one warp plays tile 1 of a two-tile scan whose tile 0 never publishes
__global__ void k_lookback_timeout(uint8_t *scratch, unsigned long long *prefix)
{
    const Lookback lb = lookback_at(scratch, 2);
    const unsigned long long e = lookback_exclusive(lb, 1, 5ull);
    if (threadIdx.x == 0) *prefix = e;
}

}  // namespace
}  // namespace gtsc

extern "C" gtsc_status gtsc_selftest_lookback_timeout(int32_t *error_word, double *seconds, void *stream)
{
    using namespace gtsc;
    if (!error_word || !seconds) return GTSC_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t *scratch = nullptr;
    const size_t bytes = lookback_bytes(2) + 16;
    if (cudaMallocAsync((void **)&scratch, bytes, s) != cudaSuccess) return GTSC_ERR_CUDA;
    gtsc_status st = GTSC_OK;
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaMemsetAsync(scratch, 0, bytes, s) != cudaSuccess) st = GTSC_ERR_CUDA;
    if (st == GTSC_OK) {
        k_lookback_timeout<<<1, 32, 0, s>>>(scratch, (unsigned long long *)(scratch + lookback_bytes(2)));
        if (cudaGetLastError() != cudaSuccess) st = GTSC_ERR_CUDA;
    }
    uint32_t err = 0;
    if (st == GTSC_OK && cudaMemcpyAsync(&err, scratch + 4, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        st = GTSC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) st = GTSC_ERR_CUDA;
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // the error word holds -status (scan.cuh records -GTSC_ERR_TIMEOUT)
    *error_word = -(int32_t)err;
    cudaFreeAsync(scratch, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) st = GTSC_ERR_CUDA;
    return st;
}
