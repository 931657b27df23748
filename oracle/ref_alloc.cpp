/*
 * ref_alloc.cpp -- device allocation and copies for the reference encoders built by
 * oracle/Makefile (target refenc).  TEST INFRASTRUCTURE ONLY.
 *
 * Those sources are compiled with cudaMalloc renamed to ref_padded_cuda_malloc and cudaMemcpy to
 * ref_cuda_memcpy, which covers their own calls (core/cuda_ptr.hpp and the encoders) and
 * Thrust's.
 *
 * Every allocation is zeroed and gets kRefPad bytes of kRefPadByte past its end.  Some reference
 * kernels read a little past a buffer: the AFL decompress kernel reads one word at the column's
 * length (compression/afl/afl_gpu.cu:172-174), and _compressUniqueKernel reads up to 32 / bits - 1
 * values past the data for the last output word (compression/unique/unique_encoding.cu:56-61).
 * With the pad those reads stay inside the allocation, and a value read from the pad matches no
 * dictionary entry (short of a column that holds the pad's bit pattern), so those last code slots
 * stay 0, as the library writes them.  Some kernels read memory they never wrote: with fewer
 * distinct values than slots, Histogram::GetMostFrequentSparse leaves the dictionary's last slots
 * unset (util/histogram/most_frequent.cu:20-22) and the dictionary coder then matches values
 * against them; zeroed memory makes those slots 0, as the library writes them.  So the reference
 * runs on the GPU without touching memory it does not own and gives the same bytes on every run.
 *
 * Every copy lets the runtime infer its direction from the pointers (cudaMemcpyDefault): the RLE
 * encoder copies its device results with cudaMemcpyHostToDevice (compression/rle/rle_encode.cu:52-53,
 * through CudaPtr::fillFromHost), which this runtime may reject as an invalid argument, and the
 * reference then exits.
 */
#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdio>

namespace {
constexpr size_t kRefPad = 4096;
constexpr int kRefPadByte = 0xA5;
}

extern "C" cudaError_t ref_padded_cuda_malloc(void **ptr, size_t size)
{
    cudaError_t e = cudaMalloc(ptr, size + kRefPad);
    if (e != cudaSuccess) return e;
    e = cudaMemset(*ptr, 0, size);
    if (e != cudaSuccess) return e;
    return cudaMemset((char *)*ptr + size, kRefPadByte, kRefPad);
}

extern "C" cudaError_t ref_cuda_memcpy(void *dst, const void *src, size_t count, enum cudaMemcpyKind kind)
{
    cudaError_t e = cudaMemcpy(dst, src, count, cudaMemcpyDefault);
    if (e != cudaSuccess) {
        // the reference exits on this error without saying which copy failed
        cudaPointerAttributes ad{}, as{};
        cudaPointerGetAttributes(&ad, dst);
        cudaPointerGetAttributes(&as, src);
        cudaGetLastError();
        fprintf(stderr, "ref_cuda_memcpy: %s: dst %p (memory type %d) src %p (memory type %d) count %zu kind %d\n",
                cudaGetErrorString(e), dst, (int)ad.type, src, (int)as.type, count, (int)kind);
    }
    return e;
}
