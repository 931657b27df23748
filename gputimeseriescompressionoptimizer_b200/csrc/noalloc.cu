// noalloc.cu -- a delta decode that allocates nothing, for callers that cannot call cudaMalloc.
//
// gtsc_decode(GTSC_DELTA, ...) allocates its output and the look-back scratch of its one-pass
// scan with cudaMallocAsync.  Some callers cannot allocate device memory: code running inside a
// host framework that owns every device allocation through its own pool, or a caller that has
// handed all device memory to another allocator.  gtsc_delta_decode_noalloc takes the output from
// the caller and keeps the scan's scratch in the file-scope array below instead.
//
// The array is reserved in every GPU that loads this library, for the life of the process.  Its
// device address is looked up with cudaGetSymbolAddress on every call, with the caller's device
// current: the lookup allocates nothing, and a cached address would go stale if the caller reset
// the device (cudaDeviceReset reloads the module, and the array can move).  The first call on a
// device also loads the library's module there, so it should come before any stream capture.
// Every call shares the array: the bytes that must start at zero are cleared at the start of each
// call, and two calls whose GPU work overlaps -- on different streams, or on different host
// threads -- race on it.
#include "kernels.hpp"
#include "scan.cuh"

namespace gtsc {

namespace {

// at most 2^24 decoded values per call: 8192 scan tiles of 2048 values
constexpr uint64_t kNoAllocMaxValues = 1ull << 24;
constexpr uint64_t kNoAllocTiles = kNoAllocMaxValues / 2048;
constexpr uint64_t kNoAllocScratchBytes = lookback_bytes(kNoAllocTiles);

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch on the current device
uint8_t *scratch_for_current_device()
{
    void *p = nullptr;
    GTSC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    return (uint8_t *)p;
}

}  // namespace

}  // namespace gtsc

using namespace gtsc;

extern "C" gtsc_status gtsc_delta_decode_noalloc(int32_t dtype, const void *d_first, const void *d_deltas,
                                                uint64_t n_deltas, void *d_out, void *stream)
{
    try {
        set_last_error("");
        const int es = dtype_size(dtype);
        if (!es) fail(GTSC_ERR_ARG, "unknown data type");
        if (!d_first || !d_out || (n_deltas && !d_deltas)) fail(GTSC_ERR_ARG, "null pointer");
        const uint64_t n = n_deltas + 1;
        if (n > kNoAllocMaxValues)
            fail(GTSC_ERR_CAPACITY, "gtsc_delta_decode_noalloc: more than 2^24 values (its static scratch limit)");
        if (((uintptr_t)d_deltas % es) || ((uintptr_t)d_out & 15))
            fail(GTSC_ERR_ARG, "deltas must be aligned to the element size and the output to 16 bytes");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        uint8_t *scratch = scratch_for_current_device();
        // launch_delta_decode clears the counter, error word and tile descriptors before its kernel
        launch_delta_decode((const uint8_t *)d_deltas, n, (const uint8_t *)d_first, (uint8_t *)d_out, scratch, es, s);
        uint32_t err = 0;
        GTSC_CUDA(cudaMemcpyAsync(&err, lookback_at(scratch, delta_decode_tiles(n)).error, 4, cudaMemcpyDeviceToHost, s));
        GTSC_CUDA(cudaStreamSynchronize(s));
        if (err) fail(-(gtsc_status)err, "delta decode: device wait gave up");
        return GTSC_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    }
}
