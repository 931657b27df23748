/*
 * gtsc.h -- C ABI of the B200 column-compression library (libgtsc.so).
 *
 * Every entry point takes plain pointers and sizes, returns a gtsc_status, and runs its GPU work on
 * the given CUDA stream (a cudaStream_t passed as void*; NULL = the legacy default stream).  Device
 * buffers returned through gtsc_buffer are allocated by the library with stream-ordered
 * cudaMallocAsync and belong to the caller, who releases them with gtsc_free.  Nothing here exits
 * the process: CUDA and format errors come back as status codes (gtsc_last_error() has the text).
 *
 * Encoding and data-type codes follow the reference's enums (compression/encoding_type.hpp:17-30;
 * the DataType values live in a submodule that is not available, so the codes below are this
 * library's own and are what it writes into serialized node headers).
 */
#ifndef GTSC_H_
#define GTSC_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gtsc_status;
enum {
    GTSC_OK = 0,
    GTSC_ERR_ARG = -1,          /* bad argument (null pointer, unknown code)                */
    GTSC_ERR_TYPE = -2,         /* encoding not defined for this data type                  */
    GTSC_ERR_CAPACITY = -3,     /* output buffer too small / size above a stated maximum    */
    GTSC_ERR_FORMAT = -4,       /* corrupt or truncated compressed input                    */
    GTSC_ERR_UNSUPPORTED = -5,  /* reference entry point without a GPU counterpart          */
    GTSC_ERR_CUDA = -6,         /* CUDA runtime error                                       */
    GTSC_ERR_TIMEOUT = -7,      /* a bounded device-side wait gave up                       */
    GTSC_ERR_NO_DEVICE = -8     /* no CUDA device                                           */
};

/* DataType (reference: modules/data, unavailable) -- this library's codes */
enum { GTSC_CHAR = 0, GTSC_SHORT = 1, GTSC_INT = 2, GTSC_TIME = 3, GTSC_FLOAT = 4, GTSC_DOUBLE = 5 };

/* EncodingType -- compression/encoding_type.hpp:17-30 */
enum {
    GTSC_DELTA = 0, GTSC_AFL = 1, GTSC_SCALE = 2, GTSC_RLE = 3, GTSC_DICT = 4, GTSC_UNIQUE = 5,
    GTSC_PATCH = 6, GTSC_NONE = 7, GTSC_FLOAT_TO_INT = 8, GTSC_CONST = 9, GTSC_GFC = 10
};

typedef struct {
    void *ptr;        /* device pointer (may be NULL when bytes == 0) */
    uint64_t bytes;
} gtsc_buffer;

/* ------------------------------------------------------------------ runtime / memory */

/* Text of the last error raised on the calling thread ("" when none). */
const char *gtsc_last_error(void);
/* Library version string. */
const char *gtsc_version(void);
/* Size in bytes of one element of `dtype` (0 for an unknown code).  GetDataTypeSize. */
int32_t gtsc_dtype_size(int32_t dtype);
/* Stream-ordered device allocation / release (cudaMallocAsync / cudaFreeAsync). */
gtsc_status gtsc_malloc(void **d_ptr, uint64_t bytes, void *stream);
gtsc_status gtsc_free(void *d_ptr, void *stream);
/* Copies; `kind` 1 = host->device, 2 = device->host, 3 = device->device (cudaMemcpyKind). */
gtsc_status gtsc_memcpy(void *dst, const void *src, uint64_t bytes, int32_t kind, void *stream);
gtsc_status gtsc_stream_synchronize(void *stream);

/* ------------------------------------------------------------------ encodings */

/*
 * Encoding::Encode(SharedCudaPtr<char> data, DataType) (compression/encoding.hpp:28-47).
 * Writes out[0] = metadata, out[1..n_out-1] = encoded streams, byte-identical to the reference
 * encoder for the same input (see DESIGN.md for the documented exceptions).  Synchronises the
 * stream once to learn the data-dependent output sizes, as the reference does.
 */
gtsc_status gtsc_encode(int32_t encoding, int32_t dtype, const void *d_in, uint64_t in_bytes,
                        gtsc_buffer out[3], uint32_t *n_out, void *stream);

/* Encoding::Decode(SharedCudaPtrVector<char>, DataType) (compression/encoding.hpp:49-68). */
gtsc_status gtsc_decode(int32_t encoding, int32_t dtype, const gtsc_buffer in[3], uint32_t n_in,
                        gtsc_buffer *out, void *stream);

/* ------------------------------------------------------------------ kernel-level entry points */

/*
 * run_afl_compress_gpu<T,1> (compression/afl/afl_gpu.cu:67-73): packs n elements of an integer
 * `dtype` at bit_length bits into d_out (out_bytes = ceil(n*b / W) * sizeof(T), W = 8*sizeof(T)),
 * the FL layout of AflEncoding.  Asynchronous; d_data and d_out 16-byte aligned.
 */
gtsc_status gtsc_afl_compress_gpu(int32_t dtype, uint32_t bit_length, const void *d_data, uint64_t n,
                                  void *d_out, uint64_t out_bytes, void *stream);
/* run_afl_decompress_gpu<T,1> (afl_gpu.cu:75-81): unpacks n values; d_comp may be unaligned. */
gtsc_status gtsc_afl_decompress_gpu(int32_t dtype, uint32_t bit_length, const void *d_comp,
                                    uint64_t comp_bytes, void *d_out, uint64_t n, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GTSC_H_ */
